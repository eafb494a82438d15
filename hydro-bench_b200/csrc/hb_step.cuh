// hb_step.cuh -- device side of the handle path: the device mesh, the step
// kernels of both layouts, and the staging and setup kernels.  Shared by
// hb_solver.cu (the forward step) and hb_adjoint.cu (the reverse step).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "hb_common.cuh"
#include "hb_physics.cuh"
#include "hydrob200.h"

namespace hb {

// ---------------------------------------------------------------------------
// device mesh
// ---------------------------------------------------------------------------
enum : uint8_t { META_CODE = 0x0F, META_OWN_FIRST = 0x10, META_HAS_NB = 0x20 };

// Launch shapes.  Edge layout: the flux kernel's threads per CTA and CTAs per
// SM asked of the compiler through __launch_bounds__ (which caps registers
// per thread), and the cell kernel's CTAs per SM (it has UPDATE_THREADS
// threads).  Tile layout: the tile kernel's threads per CTA and CTAs per SM.
enum Layout : int { LAYOUT_EDGE = HB_LAYOUT_EDGE, LAYOUT_TILE = HB_LAYOUT_TILE };
struct LaunchConfig { int layout, threads, min_blocks, update_min_blocks; };
constexpr LaunchConfig LAUNCH_CONFIGS[] = {
    {LAYOUT_EDGE, 128, 7, 8}, {LAYOUT_EDGE, 128, 6, 8}, {LAYOUT_EDGE, 128, 8, 8}, {LAYOUT_EDGE, 256, 3, 6},
    {LAYOUT_EDGE, 256, 4, 8}, {LAYOUT_EDGE, 128, 7, 6}, {LAYOUT_EDGE, 256, 2, 6}, {LAYOUT_EDGE, 64, 12, 8},
    {LAYOUT_TILE, 256, 3, 0}, {LAYOUT_TILE, 256, 2, 0}, {LAYOUT_TILE, 128, 6, 0}, {LAYOUT_TILE, 128, 4, 0},
    {LAYOUT_TILE, 512, 1, 0}, {LAYOUT_TILE, 256, 4, 0},
    {LAYOUT_EDGE, 128, 6, 6}, {LAYOUT_EDGE, 128, 6, 9}, {LAYOUT_EDGE, 128, 7, 9}, {LAYOUT_TILE, 128, 8, 0},
    {LAYOUT_TILE, 256, 5, 0}};
constexpr int N_LAUNCH_CONFIGS = sizeof(LAUNCH_CONFIGS) / sizeof(LAUNCH_CONFIGS[0]);
constexpr int DEFAULT_EDGE_CONFIG = 0;
constexpr int DEFAULT_TILE_CONFIG = 8;
constexpr int UPDATE_THREADS = 128;

// One tile of the tile layout: a compact group of cells, contiguous in the
// device order, with its records (mirror pairs inside the tile, then every
// other real slot of its cells).
struct TileDesc { int scn, cell0, cells, rec0, npairs, nsingles; };

// Constants of one scenario of a batch (the only entry for a single mesh).
struct ScnParams {
    double hm1, hm2, jl, dt;
    int per_day, ndays;        // steps per table interval; intervals in the tables
    int cell0, cells;          // the scenario's cells in the device order
};

// Device mesh.  Cells are in reverse Cuthill-McKee order.  The flux work is a
// list of records: first the interior edges whose two slots both have code 0
// and mirror each other exactly (reciprocal neighbours, negated normal, same
// length), then every other real slot on its own.  The zero-length fourth slot
// of a triangle is no record; the cell update evaluates it.
template <class A>
struct DevMesh {
    using Policy = A;
    using R = typename A::real;
    using L = typename A::level;
    int C;                     // cells
    int per_day;               // steps per table interval (steps_per_day - 1)
    int ndays, nb, nhq;
    int npairs, nrecords;
    double hm1, hm2, jl, dt;
    R *S[2];                   // [C][4] state {H, U, V, Z}, split precision {H, U, V, H_lo};
                               // a step reads S[step & 1], writes the other
    R *W;
    const L *zbc;
    const R *fnc, *dta;        // dta: DT/AREA (variant H) or AREA (variant F)
    const R *sidex;            // variant F CFL length
    const int32_t *bcell;      // [C] row of the boundary tables, -1 = none
    const uint8_t *cmask;      // [C] bit j: slot j is a real slot
    R *slotw;                  // [4C][4] per-slot terms of the cell sums {F0, dWU, dWV, SIDE}
    double *ucoef;             // [C][UPDATE_COEF] update coefficients (update kernels with COEF only)
    // Adjoint forward rollout (fp64; set only on a copy of the mesh whose
    // step launches are captured for it, null otherwise): the cell update of
    // step t also writes the new state into checkpoint (t + 1) / ckpt_every
    // of `ckpt` ([][C][4]) when t + 1 is a multiple of ckpt_every, and, when
    // t + 1 ends on an observation, a gauge cell's new depth into row
    // (t + 1) / obs_every - 1, column gauge_of[cell], of `gauge_out`.
    double *ckpt;
    const int32_t *gauge_of;   // [C] gauge index of the cell, -1 for none
    double *gauge_out;         // [observations][ngauge]
    int ckpt_every, obs_every, ngauge;
    // records [nrecords]
    const int4 *rix;           // {a, b, sa, sb}: cell of the slot, its neighbour (-1 = none),
                               // slot 4*a+j, and for a pair the slot of b (-1 otherwise)
    uint8_t *rmeta;            // code | own_first | has_nb of slot a (code changes on breach)
    const R *rgeo;             // [nrecords][4] {COSF, SINF, SIDE, 0} of slot a
    R *f0, *f1, *f2, *f3;      // [4C] fluxes of the last step, index 4*cell + j
    const R *bqt, *bdqt;       // [ndays*nb]
    const L *bzt, *bdzt;       // [ndays*nb]
    const L *btop;             // [nb]
    const int32_t *bnhq1;      // [nb]
    const L *bzw;              // [nb*nhq]; one extra zero row at index nb
    const R *bqw;              // [nb*nhq]; one extra zero row at index nb
    uint32_t *err;
    const long long *step_ctr;
    // batches: per-CTA segment tables, one scenario per CTA
    int nscen;
    const ScnParams *scn;      // [nscen]
    const int4 *fseg;          // flux CTAs {scenario, first record, records, 1 = mirror pairs}
    const int4 *useg;          // update CTAs {scenario, first cell, cells, 0}
    // edge layout, single mesh: the flux kernel takes its CTAs' record ranges
    // in reverse order (rev_flux), so the single records at the end of the
    // list (boundary slots, whose fixed-point iterations make them the slowest)
    // start first instead of forming the launch's tail.  The cell kernel takes
    // its ranges in the opposite order of the flux kernel (batches: reversed
    // when rev_update), so it starts on the slot terms the flux kernel wrote
    // last, which are still in L2 when the mesh's terms exceed it
    int rev_flux, rev_update;
    // tile layout
    const TileDesc *tiles;     // [ntiles]
    int ntiles, max_tile_cells, max_tile_pairs;
};

struct StepIndex { int par, kt, jt; long long step; };

template <class A>
__device__ __forceinline__ StepIndex step_index(const DevMesh<A> &m, int k, int per_day, int ndays) {
    const long long step = *m.step_ctr + k;
    StepIndex si;
    si.step = step;
    si.par = (int)(step & 1);
    si.jt = (int)(step / per_day);
    si.kt = 1 + (int)(step % per_day);
    if (si.jt >= ndays) {   // beyond the boundary tables: never read past them
        if (threadIdx.x == 0) atomicOr(m.err, ERRBIT_TABLE_RANGE);
        si.jt = ndays - 1;
    }
    return si;
}

template <class R> struct Vec4 { R x, y, z, w; };
__device__ __forceinline__ Vec4<double> ld4(const double *p) {
    const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    return {a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ Vec4<float> ld4(const float *p) {
    const float4 a = *reinterpret_cast<const float4 *>(p);
    return {a.x, a.y, a.z, a.w};
}
__device__ __forceinline__ void st4(double *p, double x, double y, double z, double w) {
    *reinterpret_cast<double2 *>(p) = make_double2(x, y);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(z, w);
}
__device__ __forceinline__ void st4(float *p, float x, float y, float z, float w) {
    *reinterpret_cast<float4 *>(p) = make_float4(x, y, z, w);
}

// The same for memory known to be global, 32-byte aligned: one 256-bit access
// for fp64 records on sm_100 (half the instructions of two 16-byte ones).
// Ordered like any other access (volatile, memory clobber), so they stay
// after a dependency wait.
__device__ __forceinline__ Vec4<double> ldg4(const double *p) {
    Vec4<double> v;
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ Vec4<float> ldg4(const float *p) { return ld4(p); }
__device__ __forceinline__ void stg4(double *p, double x, double y, double z, double w) {
    st_global_f64x4(p, x, y, z, w);
}
__device__ __forceinline__ void stg4(float *p, float x, float y, float z, float w) { st4(p, x, y, z, w); }

template <class A>
__device__ __forceinline__ CellStateA<A> load_cell(const DevMesh<A> &m, int par, int c) {
    const Vec4<typename A::real> v = ldg4(m.S[par] + 4 * (size_t)c);
    const typename A::level zbc = m.zbc[c];
    if constexpr (is_split<A>::value) return {v.x, v.y, v.z, split_level<A>(v.x, v.w, zbc), zbc};
    else return {v.x, v.y, v.z, v.w, zbc};
}

// Where a step keeps the slots' terms of the cell sums between the flux and
// the update: slot s at p + 4 * (s - slot0).  Global memory (m.slotw, slot0 =
// 0) between the two kernels of the edge layout; shared memory (slot0 = the
// tile's first slot) inside the tile kernel (SMEM).
template <class R, bool SMEM = false>
struct Terms {
    R *p;
    int slot0;
    static constexpr bool smem = SMEM;
};

// the slot's terms of the cell sums (functors.cu:733-741): F0 and SIDE for
// WH = fma(SIDE, F0, WH), and the complete WU / WV increments
template <class A, class T>
__device__ __forceinline__ void store_terms(const T &t, int s, const typename A::real f[4],
                                            typename A::real side, typename A::real cs, typename A::real sn) {
    using R = typename A::real;
    const R fr1 = A::add(f[1], f[3]);
    const R slcos = A::mul(side, cs), slsin = A::mul(side, sn);
    const R dwu = A::dot(slcos, fr1, -slsin, f[2], M_WU);
    const R dwv = A::dot(slsin, fr1, slcos, f[2], M_WV);
    if constexpr (T::smem) st4(t.p + 4 * (size_t)(s - t.slot0), f[0], dwu, dwv, side);
    else stg4(t.p + 4 * (size_t)(s - t.slot0), f[0], dwu, dwv, side);
}

template <class A>
__device__ __forceinline__ void store_flux(const DevMesh<A> &m, int s, const typename A::real f[4]) {
    m.f0[s] = f[0]; m.f1[s] = f[1]; m.f2[s] = f[2]; m.f3[s] = f[3];
}

// One slot on its own: flux_slot with its boundary tables (functors.cu:47-202).
// single_core takes the slot's cell a (device order, for its table row), its
// slot sa, both cells' states and the record's code byte and geometry.
template <class A, int VARIANT, class T>
__device__ __forceinline__ void single_core(const DevMesh<A> &m, int r, int a, int sa, const CellStateA<A> &own,
                                            const CellStateA<A> &nb, uint8_t meta, const Vec4<typename A::real> &g,
                                            const StepIndex &si, const StepParams &p, int write_flux, const T &tout) {
    using R = typename A::real;
    using L = typename A::level;
    SlotInA<A> in;
    in.own = own;
    in.code = (int8_t)(meta & META_CODE);
    in.own_first = meta & META_OWN_FIRST;
    in.has_nb = meta & META_HAS_NB;
    in.nb = nb;
    in.cosj = g.x; in.sinj = g.y; in.side = g.z;
    auto fetch = [&]() {
        BoundaryInA<A> bi;
        const int row = m.bcell[a];
        if (row >= 0) {
            const size_t q = (size_t)si.jt * m.nb + row;
            bi.qt = m.bqt[q]; bi.dqt = m.bdqt[q]; bi.zt = m.bzt[q]; bi.dzt = m.bdzt[q];
            bi.top = m.btop[row]; bi.nhq1 = m.bnhq1[row];
            bi.zw = m.bzw + (size_t)row * m.nhq; bi.qw = m.bqw + (size_t)row * m.nhq;
        } else {
            bi.qt = bi.dqt = R(0); bi.zt = bi.dzt = bi.top = L(0); bi.nhq1 = 0;
            bi.zw = m.bzw + (size_t)m.nb * m.nhq; bi.qw = m.bqw + (size_t)m.nb * m.nhq;
        }
        bi.nhq = m.nhq;
        return bi;
    };
    const R cl = A::sqrt(A::mul(A::c(9.81), in.own.h));
    SlotOut<R> o;
    flux_slot<A, VARIANT>(in, cl, p, fetch, o);
    if (o.mask != 0xF) {   // codes that leave fluxes unwritten keep the old values (functors.cu:525-565)
        if (!(o.mask & 1)) o.f[0] = m.f0[sa];
        if (!(o.mask & 2)) o.f[1] = m.f1[sa];
        if (!(o.mask & 4)) o.f[2] = m.f2[sa];
        if (!(o.mask & 8)) o.f[3] = m.f3[sa];
    }
    if (write_flux || o.mask != 0xF) store_flux(m, sa, o.f);
    store_terms<A>(tout, sa, o.f, in.side, in.cosj, in.sinj);
    if (o.klas_to_zero) m.rmeta[r] = (uint8_t)((meta & ~META_CODE) | CODE_ZERO);
    if (o.undefined) atomicOr(m.err, ERRBIT_UNDEFINED);
}

template <class A, int VARIANT, class T>
__device__ __forceinline__ void single_record(const DevMesh<A> &m, int r, const StepIndex &si,
                                              const StepParams &p, int write_flux, const T &tout) {
    using R = typename A::real;
    using L = typename A::level;
    const int4 ix = m.rix[r];
    const Vec4<R> g = ldg4(m.rgeo + 4 * (size_t)r);
    const uint8_t meta = m.rmeta[r];
    const CellStateA<A> own = load_cell(m, si.par, ix.x);
    const CellStateA<A> nb =
        (meta & META_HAS_NB) ? load_cell(m, si.par, ix.y) : CellStateA<A>{R(0), R(0), R(0), L(0), L(0)};
    single_core<A, VARIANT>(m, r, ix.x, ix.z, own, nb, meta, g, si, p, write_flux, tout);
}

// The mirrored Osher of a pair computed on its own (when its inputs differ
// from the direct route's in the normal velocity); mirror_core takes the
// pair's cells a (direct side) and b, its geometry and b's slot sb.
template <class A, class T>
__device__ __forceinline__ void mirror_core(const DevMesh<A> &m, const CellStateA<A> &A_, const CellStateA<A> &B_,
                                            const Vec4<typename A::real> &g, int sb, const StepParams &p,
                                            int write_flux, const T &tout) {
    using R = typename A::real;
    const R cs = g.x, sn = g.y;
    const R clA = A::sqrt(A::mul(A::c(9.81), A_.h));
    const OsherIn<R> oi = osher_inputs<A>(A_, B_, cs, sn, clA, true, p);
    R fo[4], fb[4];
    osher<A>(oi.cl, oi.ql, oi.qr, oi.fil, fo);
    fb[0] = -fo[0];
    fb[1] = osher_f1<A>(fo[1], oi.ratio, oi.hcR, oi.ur);
    fb[2] = fo[2];
    fb[3] = mirror_f3<A>(fo[3], A_.zbc, B_.zbc);
    if (write_flux) store_flux(m, sb, fb);
    store_terms<A>(tout, sb, fb, g.z, -cs, -sn);
}

template <class A, class T>
__device__ __forceinline__ void pair_mirror(const DevMesh<A> &m, int r, const StepIndex &si,
                                            const StepParams &p, int write_flux, const T &tout) {
    using R = typename A::real;
    const int4 ix = m.rix[r];
    const Vec4<R> g = ldg4(m.rgeo + 4 * (size_t)r);
    const CellStateA<A> A_ = load_cell(m, si.par, ix.x), B_ = load_cell(m, si.par, ix.y);
    mirror_core<A>(m, A_, B_, g, ix.w, p, write_flux, tout);
}

template <class R>
__device__ __forceinline__ bool same_bits(R a, R b) {
    if constexpr (sizeof(R) == 8) return __double_as_longlong((double)a) == __double_as_longlong((double)b);
    else return __float_as_int((float)a) == __float_as_int((float)b);
}

// One mirror-pair record.  It evaluates both slots' branch chains
// (functors.cu:98-150) and, when both reach Osher, runs it once: the direct
// route at a and the mirrored route at b have the same cells, normal and
// inputs except two rotations that the reference build rounds differently.
// When those agree bit for bit the two Osher evaluations are identical, and
// the b side's FLUX2 is re-summed with its own tangent if only that differs;
// otherwise the pair goes to the CTA's queue, whose mirrored Osher
// evaluations run together after the main pass (pair_mirror).
// pair_core takes both cells' states, the geometry of a's slot and the two
// slots sa, sb; a pair whose mirrored Osher must run on its own is queued as
// record r.  tslot stores the Osher trace and the tangents of a re-summed
// FLUX2 (TRACE_VALUES values): SmemTrace, the thread's slot in shared memory
// (the edge-layout kernels, whose registers are scarce), or RegTrace
// (registers: the tile kernel, whose shared memory is).
constexpr int TRACE_VALUES = 16;
template <class R>
struct SmemTrace {   // values at p[i * stride]
    R *p;
    int stride;
    __device__ __forceinline__ void set(int i, R v) { p[i * stride] = v; }
    __device__ __forceinline__ R get(int i) const { return p[i * stride]; }
    // a value kept out of registers across a stretch of code: the volatile
    // access makes the compiler read it back instead of holding it
    __device__ __forceinline__ void park(int i, R v) { *(volatile R *)(p + i * stride) = v; }
    __device__ __forceinline__ R unpark(int i) const { return *(volatile R *)(p + i * stride); }
};
template <class R>
struct RegTrace {
    R v[TRACE_VALUES];
    __device__ __forceinline__ void set(int i, R x) { v[i] = x; }
    __device__ __forceinline__ R get(int i) const { return v[i]; }
    __device__ __forceinline__ void park(int i, R x) { v[i] = x; }
    __device__ __forceinline__ R unpark(int i) const { return v[i]; }
};

template <class A, int VARIANT, class T, class TS>
__device__ __forceinline__ void pair_core(const DevMesh<A> &m, int r, const CellStateA<A> &A_,
                                          const CellStateA<A> &B_, const Vec4<typename A::real> &g, int sa, int sb,
                                          const StepParams &p, int write_flux, const T &tout, int *queue, int *qn,
                                          TS &tslot) {
    using R = typename A::real;
    const int4 ix = make_int4(0, 0, sa, sb);
    const R cs = g.x, sn = g.y;
    const R clA = A::sqrt(A::mul(A::c(9.81), A_.h));
    auto nofetch = []() { return BoundaryInA<A>{}; };
    SlotInA<A> ia, ib;
    ia.own = A_; ia.nb = B_; ia.has_nb = true; ia.own_first = true; ia.code = CODE_ZERO;
    ia.cosj = cs; ia.sinj = sn; ia.side = g.z;
    ib.own = B_; ib.nb = A_; ib.has_nb = true; ib.own_first = false; ib.code = CODE_ZERO;
    ib.cosj = -cs; ib.sinj = -sn; ib.side = ia.side;
    // each side's branch chain; a side whose fluxes are final is written at once
    int ra_, rb_;
    {
        SlotOut<R> oa;
        ra_ = flux_chain<A, VARIANT>(ia, clA, p, nofetch, oa);   // 0 or 1 (direct)
        if (!ra_) {
            if (write_flux) store_flux(m, ix.z, oa.f);
            store_terms<A>(tout, ix.z, oa.f, g.z, cs, sn);
        }
    }
    {
        SlotOut<R> ob;
        rb_ = flux_chain<A, VARIANT>(ib, R(0), p, nofetch, ob);  // 0 or 2 (mirrored)
        if (!rb_) {
            if (write_flux) store_flux(m, ix.w, ob.f);
            store_terms<A>(tout, ix.w, ob.f, g.z, -cs, -sn);
        }
    }
    if (ra_ | rb_) {
        // the two routes' inputs differ only in QL2, UR and so QR1 (osher_inputs)
        const OsherIn<R> oi = osher_inputs<A>(A_, B_, cs, sn, clA, ra_ == 0, p);
        // Everything the epilogues take besides Osher's result is formed first
        // (same operations, same bits), so that few values stay live across
        // Osher: FLUX1's correction of each side, whether b's mirrored Osher
        // equals this one (QR1 agrees), and whether b's FLUX2 must be re-summed
        // with its own tangent (only QL2 differs; the tangents and the
        // per-piece products then wait in shared memory).
        const R ur_m = ra_ ? A::dot(B_.u, cs, B_.v, sn, M_UR1) : oi.ur;
        R qr1_m = A::mul(ur_m, oi.ratio);
        if (oi.hcR <= A::c(p.hm2) || oi.qr[0] <= A::c(p.hm2)) qr1_m = A::copysign(A::c(K::VMIN), ur_m);
        const bool b_same = rb_ && (!ra_ || same_bits(oi.qr[1], qr1_m));
        const R ql2_m = ra_ ? A::dot(A_.v, cs, -A_.u, sn, M_QL2M) : oi.ql[2];
        const bool b_resum = b_same && ra_ && !same_bits(oi.ql[2], ql2_m);
        if (b_resum) { tslot.set(6, ql2_m); tslot.set(7, oi.qr[2]); }
        // the epilogues' other inputs wait across Osher in the trace store too
        // (read back afterwards rather than held in registers)
        tslot.park(8, osher_f1_term<A>(oi.ratio, oi.hcR, oi.ur));   // FLUX1 term of side a
        tslot.park(9, osher_f1_term<A>(oi.ratio, oi.hcR, ur_m));    // FLUX1 term of side b
        tslot.park(10, cs);
        tslot.park(11, sn);
        tslot.park(12, g.z);
        using L = typename A::level;
        L zbcA = A_.zbc, zbcB = B_.zbc;
        if constexpr (std::is_same<L, R>::value) { tslot.park(13, zbcA); tslot.park(14, zbcB); }
        // the two slot indices wait in the trace store too (fp64: one 64-bit slot)
        int psa = ix.z, psb = ix.w;
        if constexpr (sizeof(R) == 8)
            tslot.park(15, __longlong_as_double((long long)(((unsigned long long)(unsigned)psb << 32) | (unsigned)psa)));
        R fo[4];
        OsherTraceIn<TS> tr{&tslot, 0u, 0u};
        osher<A>(oi.cl, oi.ql, oi.qr, oi.fil, fo, &tr);
        const R pcs = tslot.unpark(10), psn = tslot.unpark(11), pside = tslot.unpark(12);
        if constexpr (std::is_same<L, R>::value) { zbcA = tslot.unpark(13); zbcB = tslot.unpark(14); }
        if constexpr (sizeof(R) == 8) {
            const unsigned long long w = (unsigned long long)__double_as_longlong((double)tslot.unpark(15));
            psa = (int)(unsigned)(w & 0xFFFFFFFFull);
            psb = (int)(unsigned)(w >> 32);
        }
        if (ra_) {
            R f[4];
            f[0] = fo[0];
            f[1] = A::add(fo[1], tslot.unpark(8));
            f[2] = fo[2];
            f[3] = fo[3];
            if (write_flux) store_flux(m, psa, f);
            store_terms<A>(tout, psa, f, pside, pcs, psn);
        }
        if (b_same) {
            R f[4];
            f[0] = -fo[0];
            f[1] = A::add(fo[1], tslot.unpark(9));
            f[2] = b_resum ? osher_f2<A>(tr, tslot.get(6), tslot.get(7)) : fo[2];
            f[3] = mirror_f3<A>(fo[3], zbcA, zbcB);
            if (write_flux) store_flux(m, psb, f);
            store_terms<A>(tout, psb, f, pside, -pcs, -psn);
        } else if (rb_) {
            queue[atomicAdd(qn, 1)] = r;
        }
    }
}

template <class A, int VARIANT, class T, class TS>
__device__ __forceinline__ void pair_record(const DevMesh<A> &m, int r, const StepIndex &si, const StepParams &p,
                                            int write_flux, const T &tout, int *queue, int *qn, TS &tslot) {
    using R = typename A::real;
    const int4 ix = m.rix[r];
    const Vec4<R> g = ldg4(m.rgeo + 4 * (size_t)r);
    const CellStateA<A> A_ = load_cell(m, si.par, ix.x), B_ = load_cell(m, si.par, ix.y);
    pair_core<A, VARIANT>(m, r, A_, B_, g, ix.z, ix.w, p, write_flux, tout, queue, qn, tslot);
}

// Flux of every record of one step.  Single mesh (SEG = false): records
// [0, npairs) are mirror pairs and the rest single slots, one per thread.
// Batch (SEG = true): CTA b takes the scenario and record range of fseg[b].
// SMEM_TRACE: the Osher trace in shared memory (fewer registers, more shared
// memory per CTA) or in registers.
template <class A, int VARIANT, int THREADS, int MINB, bool SEG, bool SMEM_TRACE = true>
__global__ void __launch_bounds__(THREADS, MINB) flux_kernel(DevMesh<A> m, int k, int write_flux) {
    using R = typename A::real;
    __shared__ int queue[THREADS];
    __shared__ int qn;
    __shared__ R trace[SMEM_TRACE ? TRACE_VALUES * THREADS : 1];
    auto tslot = [&]() {
        if constexpr (SMEM_TRACE) return SmemTrace<R>{trace + threadIdx.x, THREADS};
        else return RegTrace<R>{};
    }();
    if (threadIdx.x == 0) qn = 0;
    int r;
    bool valid, pair;
    StepIndex si;
    StepParams p;
    if constexpr (SEG) {
        const int4 d = m.fseg[blockIdx.x];   // constant tables: read before the dependency wait
        const ScnParams sp = m.scn[d.x];
        cudaGridDependencySynchronize();
        cudaTriggerProgrammaticLaunchCompletion();
        si = step_index(m, k, sp.per_day, sp.ndays);
        p = StepParams{sp.hm1, sp.hm2, sp.jl, sp.dt, si.kt, si.jt};
        r = d.y + (int)threadIdx.x;
        valid = (int)threadIdx.x < d.z;
        pair = d.w != 0;
    } else {
        cudaGridDependencySynchronize();
        cudaTriggerProgrammaticLaunchCompletion();
        si = step_index(m, k, m.per_day, m.ndays);
        p = StepParams{m.hm1, m.hm2, m.jl, m.dt, si.kt, si.jt};
        r = (m.rev_flux ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x) * THREADS + threadIdx.x;
        valid = r < m.nrecords;
        pair = r < m.npairs;
    }
    __syncthreads();
    const Terms<typename A::real> tout{m.slotw, 0};
    if (valid) {
        if (pair) pair_record<A, VARIANT>(m, r, si, p, write_flux, tout, queue, &qn, tslot);
        else single_record<A, VARIANT>(m, r, si, p, write_flux, tout);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < qn; i += THREADS) pair_mirror<A>(m, queue[i], si, p, write_flux, tout);
}

// Sums and update of one cell (UpdateCellKernel, functors.cu:717-784).  The
// zero-length fourth slot of a triangle is evaluated here, without pow
// (flux_slot's ZERO_LEN) unless fluxes are written out, and only where its
// zero addends can change the sums.
// SMEM_TERMS: `terms` is in shared memory (tile layout), else global.
// update_core takes the cell's stored state record `raw` and bed `zbc`.
template <class A, int VARIANT, bool COEF = false, bool SMEM_TERMS = false>
__device__ __forceinline__ void update_core(const DevMesh<A> &m, int c, const Vec4<typename A::real> &raw,
                                            typename A::level zbc, const StepIndex &si, const StepParams &p,
                                            int write_flux, const typename A::real *terms) {
    using R = typename A::real;
    using L = typename A::level;
    CellStateA<A> st;
    st.h = raw.x; st.u = raw.y; st.v = raw.z; st.zbc = zbc;
    if constexpr (is_split<A>::value) st.z = split_level<A>(raw.x, raw.w, st.zbc);
    else st.z = raw.w;
    const unsigned mask = m.cmask[c];
    const R fnc = m.fnc[c], dta = m.dta[c], sidex = VARIANT == 1 ? m.sidex[c] : R(0);
    // only the real slots' terms are read (a triangle's zero-length fourth
    // slot is evaluated below and has none)
    Vec4<R> t[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        t[j] = !(mask & (1u << j)) ? Vec4<R>{R(0), R(0), R(0), R(0)}
                                   : (SMEM_TERMS ? ld4(terms + 4 * j) : ldg4(terms + 4 * j));
    // The slot sums in slot order j = 0..3.  A zero-length slot (a
    // triangle's fourth) adds SIDE*F0 = 0*F0 to WH and 0*(...) to WU and WV.
    // For a finite state (h > 0) its fluxes are finite, so each addend is a
    // zero and leaves a non-zero partial sum unchanged bit for bit: the first
    // pass skips such slots.  Only a zero partial sum at a zero-length slot
    // (whose sign the addend may change), a non-finite state, or the last
    // step of a sequence (which writes the slot's fluxes) needs the slot's
    // flux: the second pass then evaluates it once (every zero-length slot of
    // a cell has the same inputs: the cell's state, no neighbour, zero
    // geometry and code 0) and redoes the sums with every slot in order.
    // Keeping that evaluation off the common path keeps the kernel's
    // register count that of the sums and the update.
    R wh = R(0), wu = R(0), wv = R(0);
    const bool finite_state = st.h > R(0) && isfinite((double)st.h) && isfinite((double)st.u) &&
                              isfinite((double)st.v) && isfinite((double)st.z) && isfinite((double)st.zbc);
    bool need_zero = false;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (mask & (1u << j)) {
            // F0 and SIDE for WH; the WU/WV increments were formed by the flux kernel
            wh = A::madd(t[j].w, t[j].x, wh, M_WH);
            wu = A::add(wu, t[j].y);
            wv = A::add(wv, t[j].z);
        } else if (write_flux || !finite_state || wh == R(0) || wu == R(0) || wv == R(0)) {
            need_zero = true;
        }
    }
    if (need_zero) {
        SlotInA<A> in;
        in.own = st;
        in.nb = {R(0), R(0), R(0), L(0), L(0)};
        in.has_nb = false; in.own_first = false; in.code = CODE_ZERO;
        in.cosj = R(0); in.sinj = R(0); in.side = R(0);
        auto nofetch = []() { return BoundaryInA<A>{}; };
        SlotOut<R> o;
        if (write_flux) {
            flux_slot<A, VARIANT, decltype(nofetch), false>(in, A::sqrt(A::mul(A::c(9.81), st.h)), p, nofetch, o);
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (!(mask & (1u << j))) store_flux(m, 4 * c + j, o.f);
        } else {
            flux_chain<A, VARIANT, decltype(nofetch), true>(in, R(0), p, nofetch, o);
        }
        wh = R(0); wu = R(0); wv = R(0);
#pragma unroll 1
        for (int j = 0; j < 4; j++) {
            if (mask & (1u << j)) {
                const Vec4<R> tj = SMEM_TERMS ? ld4(terms + 4 * j) : ldg4(terms + 4 * j);
                wh = A::madd(tj.w, tj.x, wh, M_WH);
                wu = A::add(wu, tj.y);
                wv = A::add(wv, tj.z);
            } else {
                // zero-length slot: SIDE = SLCOS = SLSIN = 0 (mesh.cpp:293-306, :347-370)
                wsum_add<A>(wh, wu, wv, o.f[0], o.f[1], o.f[2], o.f[3], R(0), R(0), R(0));
            }
        }
    }
    CellUpdateIn<R, L> ci;
    ci.h = st.h; ci.u = st.u; ci.v = st.v; ci.zbc = st.zbc;
    ci.hlo = is_split<A>::value ? raw.w : R(0);
    ci.fnc = fnc;
    ci.dta_or_area = dta;
    ci.sidex = sidex;
    CellUpdateOut<R, L> o =
        update_cell<A, VARIANT, COEF>(ci, wh, wu, wv, p, COEF ? m.ucoef + UPDATE_COEF * (size_t)c : nullptr);
    const int np = si.par ^ 1;
    if constexpr (is_split<A>::value) stg4(m.S[np] + 4 * (size_t)c, o.h, o.u, o.v, o.hlo);
    else stg4(m.S[np] + 4 * (size_t)c, o.h, o.u, o.v, o.z);
    m.W[c] = o.w;
    if (!(isfinite((double)o.h) && isfinite((double)o.u) && isfinite((double)o.v))) atomicOr(m.err, ERRBIT_NONFINITE);
    if constexpr (std::is_same<A, F64Exact>::value) {
        if (m.ckpt != nullptr) {
            const long long t1 = si.step + 1;
            if (t1 % m.ckpt_every == 0)
                stg4(m.ckpt + 4 * ((size_t)(t1 / m.ckpt_every) * (size_t)m.C + (size_t)c), o.h, o.u, o.v, o.z);
        }
        if (m.gauge_of != nullptr) {
            const long long t1 = si.step + 1;
            const int g = m.gauge_of[c];
            if (g >= 0 && t1 % m.obs_every == 0) m.gauge_out[(size_t)(t1 / m.obs_every - 1) * m.ngauge + g] = o.h;
        }
    }
}

template <class A, int VARIANT, bool COEF = false, bool SMEM_TERMS = false>
__device__ __forceinline__ void update_one(const DevMesh<A> &m, int c, const StepIndex &si, const StepParams &p,
                                           int write_flux, const typename A::real *terms) {
    const Vec4<typename A::real> raw = ldg4(m.S[si.par] + 4 * (size_t)c);
    update_core<A, VARIANT, COEF, SMEM_TERMS>(m, c, raw, m.zbc[c], si, p, write_flux, terms);
}

// Every cell of one step.  Single mesh: a grid-stride loop over the cells.
// Batch: CTA b takes the scenario and cell range of useg[b].  COEF: also the
// update coefficients of the wet cells into m.ucoef.
template <class A, int VARIANT, int UMINB, bool SEG, bool COEF = false>
__global__ void __launch_bounds__(UPDATE_THREADS, UMINB) update_kernel(DevMesh<A> m, int k, int write_flux) {
    // batches: the flux segments run forward, so the cells run reversed
    const bool rev = SEG ? m.rev_update != 0 : m.rev_flux == 0;
    const int blk = rev ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    if constexpr (SEG) {
        const int4 d = m.useg[blk];
        const ScnParams sp = m.scn[d.x];
        cudaGridDependencySynchronize();
        cudaTriggerProgrammaticLaunchCompletion();
        const StepIndex si = step_index(m, k, sp.per_day, sp.ndays);
        const StepParams p{sp.hm1, sp.hm2, sp.jl, sp.dt, si.kt, si.jt};
        const int c = d.y + (int)threadIdx.x;
        if ((int)threadIdx.x < d.z) update_one<A, VARIANT, COEF>(m, c, si, p, write_flux, m.slotw + 16 * (size_t)c);
    } else {
        cudaGridDependencySynchronize();
        cudaTriggerProgrammaticLaunchCompletion();
        const StepIndex si = step_index(m, k, m.per_day, m.ndays);
        const StepParams p{m.hm1, m.hm2, m.jl, m.dt, si.kt, si.jt};
        for (int c = blk * UPDATE_THREADS + threadIdx.x; c < m.C; c += gridDim.x * UPDATE_THREADS)
            update_one<A, VARIANT, COEF>(m, c, si, p, write_flux, m.slotw + 16 * (size_t)c);
    }
}

// The whole step of one tile (tile layout): every record of the tile writes
// its slots' terms into shared memory, then each cell of the tile sums its
// four slots in order and is updated.  Slots of edges that leave the tile are
// single records, computed by each tile for its own slot as the reference
// computes every slot; the state of the neighbour across is read from global
// memory, where the previous step (the previous launch) left it.
template <class A, int VARIANT, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) tile_kernel(DevMesh<A> m, int k, int write_flux) {
    using R = typename A::real;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    R *terms = reinterpret_cast<R *>(tile_smem);                                       // [max cells][4 slots][4]
    int *queue = reinterpret_cast<int *>(tile_smem + 16 * sizeof(R) * (size_t)m.max_tile_cells);
    __shared__ int qn;
    const TileDesc td = m.tiles[blockIdx.x];   // constant tables: read before the dependency wait
    const ScnParams sp = m.scn[td.scn];
    if (threadIdx.x == 0) qn = 0;
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
    const StepIndex si = step_index(m, k, sp.per_day, sp.ndays);
    const StepParams p{sp.hm1, sp.hm2, sp.jl, sp.dt, si.kt, si.jt};
    const Terms<R, true> tout{terms, 4 * td.cell0};
    __syncthreads();
    const int nrec = td.npairs + td.nsingles;
    for (int i = threadIdx.x; i < nrec; i += THREADS) {
        RegTrace<R> tslot;
        if (i < td.npairs) pair_record<A, VARIANT>(m, td.rec0 + i, si, p, write_flux, tout, queue, &qn, tslot);
        else single_record<A, VARIANT>(m, td.rec0 + i, si, p, write_flux, tout);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < qn; i += THREADS) pair_mirror<A>(m, queue[i], si, p, write_flux, tout);
    __syncthreads();
    for (int c = threadIdx.x; c < td.cells; c += THREADS)
        update_one<A, VARIANT, false, true>(m, td.cell0 + c, si, p, write_flux, terms + 16 * c);
}

// ---------------------------------------------------------------------------
// persistent step sequence (edge layout, hb_options.persistent)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Backstop of a barrier wait when the global timer does not advance: each
// poll is an L2 round trip (>= 0.3 us), so this many polls last >= 10 s.
constexpr unsigned BARRIER_MAX_POLLS = 1u << 25;

// Grid-wide barrier of a cooperative launch.  bar[0] counts CTA arrivals
// since the launch began and bar[1] is the launch's give-up flag (the host
// zeroes both before each launch); a barrier returns once `target` arrivals
// are counted.  The wait is bounded: after limit_ns of the global timer (or
// BARRIER_MAX_POLLS polls), or as soon as another CTA of this launch has given
// up, it raises the flag and the sticky ERRBIT_BARRIER (which hb_sync reports)
// and returns false, and the caller's CTA leaves the kernel, so a barrier that
// cannot complete ends the launch with a status instead of a hang.  The flag
// is per launch, so an error bit left by an earlier launch (or restored from
// a checkpoint) does not end later launches.  Ordering is the grid-sync
// pattern: the CTA's writes are ordered before thread 0's arrival by
// __syncthreads and a device fence, and thread 0's fence after it saw the
// count orders the CTA's later reads after every arrived CTA's writes.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned target, uint32_t *err,
                                             unsigned long long limit_ns) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        __threadfence();
        unsigned seen = atomicAdd(bar, 1u) + 1u;
        if (seen < target) {
            const unsigned long long t0 = global_ns();
            for (unsigned polls = 1;; polls++) {
                __nanosleep(32);
                seen = *(volatile unsigned *)bar;
                if (seen >= target) break;
                if ((polls & 15u) == 0) {
                    const bool other_gave_up = *(volatile unsigned *)(bar + 1) != 0u;
                    if (other_gave_up || global_ns() - t0 > limit_ns || polls >= BARRIER_MAX_POLLS) {
                        atomicExch(bar + 1, 1u);
                        atomicOr(err, ERRBIT_BARRIER);
                        good = 0;
                        break;
                    }
                }
            }
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// All n steps of a sequence in one cooperative launch whose CTAs are all
// resident: per step, the flux records in chunks of THREADS (batch: the flux
// segment table's entries) over the CTAs, a grid barrier, the cells in chunks
// of UPDATE_THREADS (batch: the cell segment table's entries), and a grid
// barrier before the next step.  Each chunk runs exactly as one CTA of
// flux_kernel / update_kernel does, so the results are those of the two-kernel
// sequence bit for bit.  `phantom` adds arrivals that never come to every
// barrier (0 in use; > 0 only to exercise the bounded wait).
template <class A, int VARIANT, int THREADS, int MINB, bool SEG>
__global__ void __launch_bounds__(THREADS, MINB)
    persistent_kernel(DevMesh<A> m, int n, int nflux, int ncell, unsigned *bar, unsigned phantom,
                      unsigned long long limit_ns) {
    // The mirrored-Osher queue collects the pairs of several chunks and is run
    // when it could not take another chunk's worth, and at the end of the flux
    // phase: one block barrier per chunk instead of three.  Every queued pair
    // is run before the grid barrier, as flux_kernel runs it before it ends.
    constexpr int QCAP = 4 * THREADS;
    __shared__ int queue[QCAP];
    __shared__ int qn;
    __shared__ typename A::real trace[TRACE_VALUES * THREADS];
    SmemTrace<typename A::real> tslot{trace + threadIdx.x, THREADS};
    const Terms<typename A::real> tout{m.slotw, 0};
    unsigned arrivals = 0;
    if (threadIdx.x == 0) qn = 0;
    __syncthreads();
    auto run_queue = [&](const StepIndex &si, const StepParams &p, int wf) {   // all threads; empties the queue
        const int nq = qn;
        for (int i = threadIdx.x; i < nq; i += THREADS) pair_mirror<A>(m, queue[i], si, p, wf, tout);
        __syncthreads();
        if (threadIdx.x == 0) qn = 0;
        __syncthreads();
    };
    for (int k = 0; k < n; k++) {
        const int wf = k == n - 1;
        StepIndex si0{};
        StepParams p0{};
        if constexpr (!SEG) {
            si0 = step_index(m, k, m.per_day, m.ndays);
            p0 = StepParams{m.hm1, m.hm2, m.jl, m.dt, si0.kt, si0.jt};
        }
        for (int b = blockIdx.x; b < nflux; b += gridDim.x) {
            int r0, cnt;
            bool seg_pairs = false;
            StepIndex si = si0;
            StepParams p = p0;
            if constexpr (SEG) {
                const int4 d = m.fseg[b];
                const ScnParams sp = m.scn[d.x];
                si = step_index(m, k, sp.per_day, sp.ndays);
                p = StepParams{sp.hm1, sp.hm2, sp.jl, sp.dt, si.kt, si.jt};
                r0 = d.y;
                cnt = d.z;
                seg_pairs = d.w != 0;
            } else {
                r0 = (m.rev_flux ? nflux - 1 - b : b) * THREADS;   // boundary singles first, as flux_kernel
                cnt = min(THREADS, m.nrecords - r0);
            }
            if ((int)threadIdx.x < cnt) {
                const int r = r0 + (int)threadIdx.x;
                const bool pair = SEG ? seg_pairs : r < m.npairs;
                if (pair) pair_record<A, VARIANT>(m, r, si, p, wf, tout, queue, &qn, tslot);
                else single_record<A, VARIANT>(m, r, si, p, wf, tout);
            }
            __syncthreads();   // the queue's count is complete
            // a batch chunk's pairs have their scenario's parameters: its queue
            // runs at once; a single mesh's when another chunk might not fit
            if (SEG || qn > QCAP - THREADS) run_queue(si, p, wf);
        }
        if constexpr (!SEG) run_queue(si0, p0, wf);
        arrivals += gridDim.x;
        if (!grid_barrier(bar, arrivals + phantom, m.err, limit_ns)) return;
        for (int b = blockIdx.x; b < ncell; b += gridDim.x) {
            int c0, cnt;
            StepIndex si;
            StepParams p;
            if constexpr (SEG) {
                const int4 d = m.useg[b];
                const ScnParams sp = m.scn[d.x];
                si = step_index(m, k, sp.per_day, sp.ndays);
                p = StepParams{sp.hm1, sp.hm2, sp.jl, sp.dt, si.kt, si.jt};
                c0 = d.y;
                cnt = d.z;
            } else {
                si = step_index(m, k, m.per_day, m.ndays);
                p = StepParams{m.hm1, m.hm2, m.jl, m.dt, si.kt, si.jt};
                c0 = b * UPDATE_THREADS;
                cnt = min(UPDATE_THREADS, m.C - c0);
            }
            for (int i = threadIdx.x; i < cnt; i += THREADS)
                update_one<A, VARIANT>(m, c0 + i, si, p, wf, m.slotw + 16 * (size_t)(c0 + i));
        }
        if (k + 1 < n) {
            arrivals += gridDim.x;
            if (!grid_barrier(bar, arrivals + phantom, m.err, limit_ns)) return;
        }
    }
}

// Advances the step counter after a step sequence.  Launched with
// programmatic dependent launch like the step kernels: it waits for the last
// step's results and lets the next kernel launch at once.
static __global__ void tick_kernel(long long *ctr, int n) {
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
    *ctr += n;
}

// Split precision state <-> the reference's (H, Z) of one cell.  The depth is
// kept as the fp32 pair (h, hlo) with h + hlo = H; a cell at or below the dry
// threshold keeps in hlo the offset of its level instead (split_level).
struct SplitCodec {
    static __host__ __device__ inline void encode(double H, double Z, double zbc, float hm1f, float &h, float &hlo) {
        h = (float)H;
        hlo = h > hm1f ? (float)(H - (double)h) : (float)((Z - zbc) - (double)h);
    }
    static __host__ __device__ inline double depth(float h, float hlo, float hm1f, double hm1) {
        return h > hm1f ? (double)h + (double)hlo : (h == hm1f ? hm1 : (double)h);
    }
    static __host__ __device__ inline double level(float h, float hlo, double zbc) {
        return (double)h + ((double)hlo + zbc);
    }
};

// Reference-order staging <-> device-order state of one scenario: cells
// [cell0, cell0 + C) of the device state, perm[new] = old within the scenario.
template <class A>
__global__ void stage_in_kernel(DevMesh<A> m, int cell0, int C, double hm1, const int32_t *__restrict__ perm,
                                const double *__restrict__ stage) {
    using R = typename A::real;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    const int o = perm[i];
    R *d = m.S[(*m.step_ctr) & 1] + 4 * ((size_t)cell0 + i);
    d[1] = (R)stage[(size_t)C + o];
    d[2] = (R)stage[2 * (size_t)C + o];
    if constexpr (is_split<A>::value) {
        float h, hlo;
        SplitCodec::encode(stage[o], stage[3 * (size_t)C + o], m.zbc[cell0 + i], (float)hm1, h, hlo);
        d[0] = h; d[3] = hlo;
    } else {
        d[0] = (R)stage[o];
        d[3] = (R)stage[3 * (size_t)C + o];
    }
}
template <class A>
__global__ void stage_out_kernel(DevMesh<A> m, int cell0, int C, double hm1, const int32_t *__restrict__ perm,
                                 double *__restrict__ stage) {
    using R = typename A::real;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    const int o = perm[i];
    const R *d = m.S[(*m.step_ctr) & 1] + 4 * ((size_t)cell0 + i);
    stage[(size_t)C + o] = (double)d[1];
    stage[2 * (size_t)C + o] = (double)d[2];
    if constexpr (is_split<A>::value) {
        stage[o] = SplitCodec::depth(d[0], d[3], (float)hm1, hm1);
        stage[3 * (size_t)C + o] = SplitCodec::level(d[0], d[3], m.zbc[cell0 + i]);
    } else {
        stage[o] = (double)d[0];
        stage[3 * (size_t)C + o] = (double)d[3];
    }
    stage[4 * (size_t)C + o] = (double)m.W[cell0 + i];
}

// per-cell constants that the update needs, computed on the device with the
// reference's arithmetic (functors.cu:750, v0 functors.cu:752-763)
template <class A, int VARIANT>
__global__ void setup_cells_kernel(int C, double dt, const typename A::real *area, const typename A::real *side4,
                                   typename A::real *dta, typename A::real *sidex) {
    using R = typename A::real;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    if (VARIANT == 1) {
        const R s0 = side4[4 * i], s1 = side4[4 * i + 1], s2 = side4[4 * i + 2], s3 = side4[4 * i + 3];
        if (s3 > R(0)) sidex[i] = A::fmin(A::mul(A::c(0.5), A::add(s0, s2)), A::mul(A::c(0.5), A::add(s1, s3)));
        else {
            R ss = A::mul(A::c(0.5), A::add(A::add(s0, s1), s2));
            sidex[i] = A::sqrt(A::div(A::mul(A::mul(A::sub(ss, s0), A::sub(ss, s1)), A::sub(ss, s2)), ss));
        }
        dta[i] = area[i];
    } else {
        dta[i] = A::div(A::c(dt), area[i]);
    }
}

}  // namespace hb
