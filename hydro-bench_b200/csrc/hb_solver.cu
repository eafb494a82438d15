// hb_solver.cu -- the handle-based path: the mesh lives on the device in a
// bandwidth-reduced cell order, and one kernel launch per step computes every
// slot's flux and the cell update together.
//
// Step kernel layout: four consecutive lanes of a warp own the four slots of
// one cell (slot j on lane 4*c + j).  Each lane computes its slot's flux
// (CalculateFluxKernel, functors.cu:47-202), the four lanes exchange their
// fluxes with warp shuffles and sum them in slot order j = 0..3 (the order of
// UpdateCellKernel, functors.cu:732-742), and lane j = 0 writes the cell's new
// state (functors.cu:744-783).  The state is double-buffered: a step reads
// buffer (step & 1) and writes the other, which is what the reference's
// two-kernel sequence amounts to.  The per-slot flux arrays are written only
// by the last step of a launch sequence, plus every step for the slots whose
// boundary code leaves some fluxes unwritten (those keep their old values,
// functors.cu:525-565).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include "hb_common.cuh"
#include "hb_physics.cuh"
#include "hydrob200.h"

// ---------------------------------------------------------------------------
// error reporting
// ---------------------------------------------------------------------------
namespace {
thread_local int t_last_status = HB_OK;
thread_local char t_last_msg[512] = "";
}  // namespace

namespace hb {
int set_error(int status, const char *fmt, ...) {
    t_last_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_last_msg, sizeof t_last_msg, fmt, ap);
    va_end(ap);
    return status;
}
}  // namespace hb

extern "C" int hb_last_error(void) { return t_last_status; }
extern "C" const char *hb_last_error_string(void) { return t_last_msg; }
extern "C" const char *hb_status_string(int s) {
    switch (s) {
    case HB_OK: return "ok";
    case HB_E_INVALID: return "invalid argument";
    case HB_E_BADMESH: return "inconsistent mesh";
    case HB_E_CUDA: return "CUDA error";
    case HB_E_NONFINITE: return "non-finite state";
    case HB_E_BARRIER_TIMEOUT: return "grid barrier timeout";
    case HB_E_IO: return "deck file error";
    case HB_E_UNDEFINED_REF: return "slot reached undefined reference behaviour";
    case HB_E_NOMEM: return "out of memory";
    case HB_E_TOO_LARGE: return "size beyond capacity";
    default: return "unknown status";
    }
}

extern "C" void hb_options_default(hb_options *o) {
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->variant = HB_VARIANT_H;
    o->precision = HB_FP64;
    o->device = 0;
    o->renumber = 1;
    o->tile_config = 0;
}

namespace hb {

// ---------------------------------------------------------------------------
// device mesh
// ---------------------------------------------------------------------------
enum : uint8_t { META_CODE = 0x0F, META_OWN_FIRST = 0x10, META_HAS_NB = 0x20 };

// Tile configurations of the step kernel: threads per CTA (= the most real
// slots and the most cells a tile holds) and the CTAs per SM the compiler is
// asked to fit (__launch_bounds__), which caps the registers per thread.
struct TileConfig { int threads, min_blocks; };
constexpr TileConfig TILE_CONFIGS[] = {{256, 2}, {256, 3}, {256, 4}, {128, 6}, {128, 8}, {512, 2}};
constexpr int N_TILE_CONFIGS = sizeof(TILE_CONFIGS) / sizeof(TILE_CONFIGS[0]);
constexpr int DEFAULT_TILE_CONFIG = 2;   // (256, 4): fastest in the 207,234-cell sweep

// Device mesh.  Cells are in reverse Cuthill-McKee order and cut into tiles of
// consecutive cells holding at most TILE real slots; a tile is one CTA.  Real
// slots (every slot except the zero-length fourth slot of a triangle) are
// stored compactly, tile by tile, in slot order within each cell.
template <class R>
struct DevMesh {
    int C;                     // cells
    int per_day;               // steps per table interval (steps_per_day - 1)
    int ndays, nb, nhq, ntiles;
    double hm1, hm2, jl, dt;
    R *H[2], *U[2], *V[2], *Z[2];
    R *W;
    const R *zbc, *fnc, *dta;  // dta: DT/AREA (variant H) or AREA (variant F)
    const R *sidex;            // variant F CFL length
    const int32_t *bcell;      // [C] row of the boundary tables, -1 = none
    const int32_t *cslot0;     // [C] first compact slot of the cell
    const uint8_t *cmask;      // [C] bit j: slot j is a real slot
    const int32_t *tcell0;     // [ntiles+1] first cell of each tile
    const int32_t *tslot0;     // [ntiles+1] first compact slot of each tile
    // compact real slots [NS]
    const int32_t *scell;      // owning cell
    const uint8_t *sj;         // slot index j within the cell
    const int32_t *nbr;        // neighbour (device order), -1 = none
    uint8_t *meta;             // code | own_first | has_nb (code changes on breach)
    const R *cosf, *sinf, *side;
    R *f0, *f1, *f2, *f3;      // [4C] persistent fluxes, index 4*cell + j
    const R *bqt, *bdqt, *bzt, *bdzt;   // [ndays*nb]
    const R *btop;             // [nb]
    const int32_t *bnhq1;      // [nb]
    const R *bzw, *bqw;        // [nb*nhq]; one extra zero row at index nb
    uint32_t *err;
    const long long *step_ctr;
};

// One step of one tile.  Phase 1: a thread per real slot computes the slot's
// flux (CalculateFluxKernel, functors.cu:47-202) into shared memory.
// Phase 2: a thread per cell sums its four slots in order j = 0..3 and
// updates the cell (UpdateCellKernel, functors.cu:717-784); the zero-length
// fourth slot of a triangle is evaluated there, without pow (flux_slot's
// ZERO_LEN).  The state is double-buffered: read (step & 1), write the other.
template <class A, int VARIANT, int TILE, int MINB>
__global__ void __launch_bounds__(TILE, MINB) step_kernel(DevMesh<typename A::real> m, int k, int write_flux) {
    using R = typename A::real;
    __shared__ R sf[4][TILE];
    __shared__ R sg[3][TILE];
    const long long step = *m.step_ctr + k;
    const int par = (int)(step & 1);
    int jt = (int)(step / m.per_day);
    const int kt = 1 + (int)(step % m.per_day);
    if (jt >= m.ndays) {   // beyond the boundary tables: never read past them
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(m.err, ERRBIT_TABLE_RANGE);
        jt = m.ndays - 1;
    }
    const R *__restrict__ H = m.H[par];
    const R *__restrict__ U = m.U[par];
    const R *__restrict__ V = m.V[par];
    const R *__restrict__ Z = m.Z[par];
    const StepParams p{m.hm1, m.hm2, m.jl, m.dt, kt, jt};
    const int tile = blockIdx.x;
    const int t = threadIdx.x;
    const int c0 = m.tcell0[tile], c1 = m.tcell0[tile + 1];
    const int s0 = m.tslot0[tile], s1 = m.tslot0[tile + 1];

    if (s0 + t < s1) {
        const int s = s0 + t;
        const int c = m.scell[s];
        const int j = m.sj[s];
        SlotIn<R> in;
        in.own = {H[c], U[c], V[c], Z[c], m.zbc[c]};
        const uint8_t meta = m.meta[s];
        const int nb = m.nbr[s];
        in.code = (int8_t)(meta & META_CODE);
        in.own_first = meta & META_OWN_FIRST;
        in.has_nb = meta & META_HAS_NB;
        if (in.has_nb) in.nb = {H[nb], U[nb], V[nb], Z[nb], m.zbc[nb]};
        else in.nb = {R(0), R(0), R(0), R(0), R(0)};
        in.cosj = m.cosf[s];
        in.sinj = m.sinf[s];
        in.side = m.side[s];
        auto fetch = [&]() {
            BoundaryIn<R> b;
            const int r = m.bcell[c];
            if (r >= 0) {
                const size_t q = (size_t)jt * m.nb + r;
                b.qt = m.bqt[q]; b.dqt = m.bdqt[q]; b.zt = m.bzt[q]; b.dzt = m.bdzt[q];
                b.top = m.btop[r]; b.nhq1 = m.bnhq1[r];
                b.zw = m.bzw + (size_t)r * m.nhq; b.qw = m.bqw + (size_t)r * m.nhq;
            } else {
                b.qt = b.dqt = b.zt = b.dzt = b.top = R(0); b.nhq1 = 0;
                b.zw = m.bzw + (size_t)m.nb * m.nhq; b.qw = m.bqw + (size_t)m.nb * m.nhq;
            }
            b.nhq = m.nhq;
            return b;
        };
        const R cl = A::sqrt(A::mul(A::c(9.81), in.own.h));
        SlotOut<R> o;
        flux_slot<A, VARIANT>(in, cl, p, fetch, o);
        const size_t fs = 4 * (size_t)c + j;
        if (o.mask != 0xF) {   // codes that leave fluxes unwritten keep the old values
            if (!(o.mask & 1)) o.f[0] = m.f0[fs];
            if (!(o.mask & 2)) o.f[1] = m.f1[fs];
            if (!(o.mask & 4)) o.f[2] = m.f2[fs];
            if (!(o.mask & 8)) o.f[3] = m.f3[fs];
        }
        if (write_flux || in.code == CODE_BOUNDA_OTHER) {
            m.f0[fs] = o.f[0]; m.f1[fs] = o.f[1]; m.f2[fs] = o.f[2]; m.f3[fs] = o.f[3];
        }
        if (o.klas_to_zero) m.meta[s] = (uint8_t)((meta & ~META_CODE) | CODE_ZERO);
        if (o.undefined) atomicOr(m.err, ERRBIT_UNDEFINED);
        sf[0][t] = o.f[0]; sf[1][t] = o.f[1]; sf[2][t] = o.f[2]; sf[3][t] = o.f[3];
        sg[0][t] = in.side; sg[1][t] = in.cosj; sg[2][t] = in.sinj;
    }
    __syncthreads();
    if (c0 + t >= c1) return;
    const int c = c0 + t;
    const R h = H[c], u = U[c], v = V[c], z = Z[c], zbc = m.zbc[c];
    const unsigned mask = m.cmask[c];
    int q = m.cslot0[c] - s0;
    R wh = R(0), wu = R(0), wv = R(0);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        R f0, f1, f2, f3, sd, cs, sn;
        if (mask & (1u << j)) {
            f0 = sf[0][q]; f1 = sf[1][q]; f2 = sf[2][q]; f3 = sf[3][q];
            sd = sg[0][q]; cs = sg[1][q]; sn = sg[2][q];
            q++;
        } else {
            // zero-length slot without neighbour, code 0, COSF = SINF = SIDE = 0
            SlotIn<R> in;
            in.own = {h, u, v, z, zbc};
            in.nb = {R(0), R(0), R(0), R(0), R(0)};
            in.has_nb = false; in.own_first = false; in.code = CODE_ZERO;
            in.cosj = R(0); in.sinj = R(0); in.side = R(0);
            auto nofetch = []() { return BoundaryIn<R>{}; };
            const R cl = A::sqrt(A::mul(A::c(9.81), h));
            SlotOut<R> o;
            if (write_flux) {
                flux_slot<A, VARIANT, decltype(nofetch), false>(in, cl, p, nofetch, o);
                const size_t fs = 4 * (size_t)c + j;
                m.f0[fs] = o.f[0]; m.f1[fs] = o.f[1]; m.f2[fs] = o.f[2]; m.f3[fs] = o.f[3];
            } else {
                flux_slot<A, VARIANT, decltype(nofetch), true>(in, cl, p, nofetch, o);
            }
            f0 = o.f[0]; f1 = o.f[1]; f2 = o.f[2]; f3 = o.f[3];
            sd = R(0); cs = R(0); sn = R(0);
        }
        // SLCOS = SIDE*COSF, SLSIN = SIDE*SINF (mesh.cpp:368-369): one rounded product each
        wsum_add<A>(wh, wu, wv, f0, f1, f2, f3, sd, A::mul(sd, cs), A::mul(sd, sn));
    }
    CellUpdateIn<R> ci;
    ci.h = h; ci.u = u; ci.v = v; ci.zbc = zbc;
    ci.fnc = m.fnc[c];
    ci.dta_or_area = m.dta[c];
    ci.sidex = VARIANT == 1 ? m.sidex[c] : R(0);
    CellUpdateOut<R> r = update_cell<A, VARIANT>(ci, wh, wu, wv, p);
    const int np = par ^ 1;
    m.H[np][c] = r.h; m.U[np][c] = r.u; m.V[np][c] = r.v; m.Z[np][c] = r.z; m.W[c] = r.w;
    if (!(isfinite((double)r.h) && isfinite((double)r.u) && isfinite((double)r.v))) atomicOr(m.err, ERRBIT_NONFINITE);
}

__global__ void tick_kernel(long long *ctr, int n) { *ctr += n; }

// reference-order staging <-> device-order state (perm[new] = old)
template <class R>
__global__ void stage_in_kernel(int C, const int32_t *__restrict__ perm, const double *__restrict__ stage,
                                const long long *ctr, R *H0, R *U0, R *V0, R *Z0, R *H1, R *U1, R *V1, R *Z1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    const int o = perm[i];
    const bool odd = (*ctr) & 1;
    (odd ? H1 : H0)[i] = (R)stage[o];
    (odd ? U1 : U0)[i] = (R)stage[(size_t)C + o];
    (odd ? V1 : V0)[i] = (R)stage[2 * (size_t)C + o];
    (odd ? Z1 : Z0)[i] = (R)stage[3 * (size_t)C + o];
}
template <class R>
__global__ void stage_out_kernel(int C, const int32_t *__restrict__ perm, double *__restrict__ stage,
                                 const long long *ctr, const R *H0, const R *U0, const R *V0, const R *Z0,
                                 const R *H1, const R *U1, const R *V1, const R *Z1, const R *W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    const int o = perm[i];
    const bool odd = (*ctr) & 1;
    stage[o] = (double)(odd ? H1 : H0)[i];
    stage[(size_t)C + o] = (double)(odd ? U1 : U0)[i];
    stage[2 * (size_t)C + o] = (double)(odd ? V1 : V0)[i];
    stage[3 * (size_t)C + o] = (double)(odd ? Z1 : Z0)[i];
    stage[4 * (size_t)C + o] = (double)W[i];
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

// ---------------------------------------------------------------------------
// reverse Cuthill-McKee over the cell adjacency (integer-only; changes no arithmetic)
// ---------------------------------------------------------------------------
std::vector<int32_t> rcm_order(int C, const std::vector<int32_t> &nbr4) {
    std::vector<int> deg(C, 0);
    for (int i = 0; i < C; i++)
        for (int j = 0; j < 4; j++) if (nbr4[4 * i + j] >= 0) deg[i]++;
    std::vector<int32_t> order;
    order.reserve(C);
    std::vector<char> seen(C, 0);
    std::vector<int> cand(C);
    std::iota(cand.begin(), cand.end(), 0);
    std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    auto bfs_last = [&](int start, std::vector<int> &levels) {
        // returns the last node of a BFS from start (a pseudo-peripheral candidate)
        std::queue<int> q;
        std::vector<int> local;
        q.push(start);
        levels[start] = 0;
        int last = start;
        while (!q.empty()) {
            int x = q.front(); q.pop();
            local.push_back(x);
            last = x;
            for (int j = 0; j < 4; j++) {
                int y = nbr4[4 * x + j];
                if (y >= 0 && levels[y] < 0) { levels[y] = levels[x] + 1; q.push(y); }
            }
        }
        for (int x : local) levels[x] = -1;
        return last;
    };
    std::vector<int> levels(C, -1);
    for (int seed : cand) {
        if (seen[seed]) continue;
        int start = bfs_last(bfs_last(seed, levels), levels);
        size_t head = order.size();
        order.push_back(start);
        seen[start] = 1;
        while (head < order.size()) {
            int x = order[head++];
            int nb[4], n = 0;
            for (int j = 0; j < 4; j++) {
                int y = nbr4[4 * x + j];
                if (y >= 0 && !seen[y]) { nb[n++] = y; seen[y] = 1; }
            }
            std::sort(nb, nb + n, [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
            for (int q = 0; q < n; q++) order.push_back(nb[q]);
        }
    }
    std::reverse(order.begin(), order.end());
    return order;   // order[new] = old
}

}  // namespace hb

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
struct hb_handle {
    hb_options opt;
    int C = 0, ndays = 0, nhq = 0, steps_per_day = 0, per_day = 0;
    double dt = 0, hm1 = 0, hm2 = 0, jl = 0;
    std::vector<int32_t> perm;       // perm[new] = old
    std::vector<int32_t> inv;        // inv[old] = new
    std::vector<double> klas_orig;   // [4C] reference order
    std::vector<void *> allocs;
    hb::DevMesh<double> m64{};
    hb::DevMesh<float> m32{};
    uint32_t *d_err = nullptr;
    long long *d_ctr = nullptr;
    int32_t *d_perm = nullptr;       // perm on the device
    std::vector<int32_t> slot_index; // [4C] device-order slot -> compact real slot, -1 = zero-length slot
    int nslots = 0;
    int ntiles() const { return fp32() ? m32.ntiles : m64.ntiles; }
    double *d_stage = nullptr;       // [5C] reference-order staging for hb_step_host
    long long steps_done = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_steps = 0;
    int tile_config = 0;             // index into TILE_CONFIGS
    bool fp32() const { return opt.precision == HB_FP32; }
    ~hb_handle() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        for (void *p : allocs) cudaFree(p);
    }
};

namespace {

template <class T>
int dev_upload(hb_handle *h, T **dst, const std::vector<T> &src) {
    void *p = nullptr;
    size_t n = std::max<size_t>(src.size(), 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) return hb::set_error(HB_E_NOMEM, "cudaMalloc(%zu): %s", n, cudaGetErrorString(e));
    h->allocs.push_back(p);
    if (!src.empty()) HB_CUDA_RET(cudaMemcpy(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    else HB_CUDA_RET(cudaMemset(p, 0, n));
    *dst = (T *)p;
    return HB_OK;
}
template <class T>
int dev_alloc(hb_handle *h, T **dst, size_t count) {
    void *p = nullptr;
    size_t n = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) return hb::set_error(HB_E_NOMEM, "cudaMalloc(%zu): %s", n, cudaGetErrorString(e));
    h->allocs.push_back(p);
    HB_CUDA_RET(cudaMemset(p, 0, n));
    *dst = (T *)p;
    return HB_OK;
}

#define TRY(x) do { int st_ = (x); if (st_ != HB_OK) return st_; } while (0)

template <class R>
int build_device_mesh(hb_handle *h, const hb_mesh_desc *md, hb::DevMesh<R> &m) {
    const int C = h->C;
    const size_t S = 4 * (size_t)C;
    const auto &perm = h->perm;
    const auto &inv = h->inv;
    auto cellv = [&](const double *src) {
        std::vector<R> v(C);
        for (int i = 0; i < C; i++) v[i] = (R)src[perm[i]];
        return v;
    };
    auto slotv = [&](const double *src) {
        std::vector<R> v(S);
        for (int i = 0; i < C; i++)
            for (int j = 0; j < 4; j++) v[4 * (size_t)i + j] = (R)src[4 * (size_t)perm[i] + j];
        return v;
    };
    m.C = C;
    m.per_day = h->per_day;
    m.ndays = h->ndays;
    m.nhq = h->nhq;
    m.hm1 = h->hm1; m.hm2 = h->hm2; m.jl = h->jl; m.dt = h->dt;
    // real slots: everything except a zero-length slot without neighbour and code 0
    std::vector<int32_t> nbr4(S, -1);
    std::vector<uint8_t> meta4(S, 0);
    std::vector<char> real4(S, 0);
    std::vector<char> needs_table(C, 0);
    for (int i = 0; i < C; i++) {
        const int old = perm[i];
        for (int j = 0; j < 4; j++) {
            const size_t so = 4 * (size_t)old + j, sn = 4 * (size_t)i + j;
            const int nc_old = (int)(md->nac[so] - 1.0);
            int8_t code = hb::klas_code(md->klas[so]);
            uint8_t mt = (uint8_t)code;
            if (nc_old != -1) {
                if (nc_old < 0 || nc_old >= C)
                    return hb::set_error(HB_E_BADMESH, "NAC of cell %d slot %d = %g out of range", old + 1, j, md->nac[so]);
                nbr4[sn] = inv[nc_old];
                mt |= hb::META_HAS_NB;
                if (old < nc_old) mt |= hb::META_OWN_FIRST;
            }
            meta4[sn] = mt;
            real4[sn] = !(md->side[so] == 0.0 && md->cosf[so] == 0.0 && md->sinf[so] == 0.0 && nc_old == -1 &&
                          code == hb::CODE_ZERO);
            if (code == hb::CODE_K10 || code == hb::CODE_K1 || code == hb::CODE_K3 || code == hb::CODE_K6 ||
                code == hb::CODE_K7)
                needs_table[i] = 1;
        }
    }
    // tiles of consecutive cells with at most TILE real slots (and TILE cells)
    std::vector<int32_t> tcell0{0}, tslot0{0}, cslot0(C), scell, nbr;
    std::vector<uint8_t> cmask(C), sj, meta;
    std::vector<R> scos, ssin, sside;
    h->slot_index.assign(S, -1);
    int tile_slots = 0, tile_cells = 0;
    for (int i = 0; i < C; i++) {
        int nreal = 0;
        for (int j = 0; j < 4; j++) nreal += real4[4 * (size_t)i + j];
        const int TILE = hb::TILE_CONFIGS[h->tile_config].threads;
        if (tile_slots + nreal > TILE || tile_cells + 1 > TILE) {
            tcell0.push_back(i);
            tslot0.push_back((int32_t)scell.size());
            tile_slots = 0; tile_cells = 0;
        }
        cslot0[i] = (int32_t)scell.size();
        uint8_t mk = 0;
        for (int j = 0; j < 4; j++) {
            const size_t sn = 4 * (size_t)i + j, so = 4 * (size_t)perm[i] + j;
            if (!real4[sn]) continue;
            mk |= (uint8_t)(1u << j);
            h->slot_index[sn] = (int32_t)scell.size();
            scell.push_back(i); sj.push_back((uint8_t)j); nbr.push_back(nbr4[sn]); meta.push_back(meta4[sn]);
            scos.push_back((R)md->cosf[so]); ssin.push_back((R)md->sinf[so]); sside.push_back((R)md->side[so]);
        }
        cmask[i] = mk;
        tile_slots += nreal;
        tile_cells += 1;
    }
    tcell0.push_back(C);
    tslot0.push_back((int32_t)scell.size());
    m.ntiles = (int)tcell0.size() - 1;
    h->nslots = (int)scell.size();
    // compact boundary tables
    std::vector<int32_t> bcell(C, -1);
    std::vector<int> rows;
    for (int i = 0; i < C; i++) if (needs_table[i]) { bcell[i] = (int32_t)rows.size(); rows.push_back(i); }
    const int NB = (int)rows.size(), ND = h->ndays, NHQ = std::max(h->nhq, 0);
    std::vector<R> bqt((size_t)ND * NB), bdqt((size_t)ND * NB), bzt((size_t)ND * NB), bdzt((size_t)ND * NB);
    std::vector<R> btop(NB), bzw((size_t)(NB + 1) * NHQ, R(0)), bqw((size_t)(NB + 1) * NHQ, R(0));
    std::vector<int32_t> bnhq1(NB);
    for (int r = 0; r < NB; r++) {
        const int old = perm[rows[r]];
        for (int d = 0; d < ND; d++) {
            const size_t t = (size_t)d * C + old;
            bqt[(size_t)d * NB + r] = (R)md->qt[t]; bdqt[(size_t)d * NB + r] = (R)md->dqt[t];
            bzt[(size_t)d * NB + r] = (R)md->zt[t]; bdzt[(size_t)d * NB + r] = (R)md->dzt[t];
        }
        btop[r] = (R)md->bfeat[old];
        bnhq1[r] = md->nhq1[old];
        for (int q = 0; q < NHQ; q++) {
            bzw[(size_t)r * NHQ + q] = (R)md->zw[(size_t)old * NHQ + q];
            bqw[(size_t)r * NHQ + q] = (R)md->qw[(size_t)old * NHQ + q];
        }
    }
    m.nb = NB;
    const R *c;
    int32_t *ip;
    uint8_t *up;
    R *rp;
    TRY(dev_upload(h, &rp, cellv(md->zbc))); m.zbc = rp;
    TRY(dev_upload(h, &rp, cellv(md->fnc))); m.fnc = rp;
    R *area_d = nullptr, *side_d = nullptr;
    TRY(dev_upload(h, &area_d, cellv(md->area)));
    TRY(dev_upload(h, &side_d, slotv(md->side)));   // [4C], for the per-cell setup only
    TRY(dev_upload(h, &rp, sside)); m.side = rp;
    TRY(dev_upload(h, &rp, scos)); m.cosf = rp;
    TRY(dev_upload(h, &rp, ssin)); m.sinf = rp;
    TRY(dev_upload(h, &ip, nbr)); m.nbr = ip;
    TRY(dev_upload(h, &up, meta)); m.meta = up;
    TRY(dev_upload(h, &ip, scell)); m.scell = ip;
    TRY(dev_upload(h, &up, sj)); m.sj = up;
    TRY(dev_upload(h, &ip, cslot0)); m.cslot0 = ip;
    TRY(dev_upload(h, &up, cmask)); m.cmask = up;
    TRY(dev_upload(h, &ip, tcell0)); m.tcell0 = ip;
    TRY(dev_upload(h, &ip, tslot0)); m.tslot0 = ip;
    TRY(dev_upload(h, &ip, bcell)); m.bcell = ip;
    TRY(dev_upload(h, &rp, bqt)); m.bqt = rp;
    TRY(dev_upload(h, &rp, bdqt)); m.bdqt = rp;
    TRY(dev_upload(h, &rp, bzt)); m.bzt = rp;
    TRY(dev_upload(h, &rp, bdzt)); m.bdzt = rp;
    TRY(dev_upload(h, &rp, btop)); m.btop = rp;
    TRY(dev_upload(h, &ip, bnhq1)); m.bnhq1 = ip;
    TRY(dev_upload(h, &rp, bzw)); m.bzw = rp;
    TRY(dev_upload(h, &rp, bqw)); m.bqw = rp;
    for (int b = 0; b < 2; b++) {
        TRY(dev_alloc(h, &m.H[b], C)); TRY(dev_alloc(h, &m.U[b], C));
        TRY(dev_alloc(h, &m.V[b], C)); TRY(dev_alloc(h, &m.Z[b], C));
    }
    TRY(dev_alloc(h, &m.W, C));
    TRY(dev_alloc(h, &m.f0, S)); TRY(dev_alloc(h, &m.f1, S));
    TRY(dev_alloc(h, &m.f2, S)); TRY(dev_alloc(h, &m.f3, S));
    R *dta = nullptr, *sidex = nullptr;
    TRY(dev_alloc(h, &dta, C));
    TRY(dev_alloc(h, &sidex, C));
    const int blocks = (C + 255) / 256;
    using A = typename std::conditional<std::is_same<R, double>::value, hb::F64Exact, hb::F32Fast>::type;
    if (h->opt.variant == HB_VARIANT_F) hb::setup_cells_kernel<A, 1><<<blocks, 256>>>(C, h->dt, area_d, side_d, dta, sidex);
    else hb::setup_cells_kernel<A, 0><<<blocks, 256>>>(C, h->dt, area_d, side_d, dta, sidex);
    HB_CUDA_RET(cudaGetLastError());
    HB_CUDA_RET(cudaDeviceSynchronize());
    m.dta = dta;
    m.sidex = sidex;
    m.err = h->d_err;
    m.step_ctr = h->d_ctr;
    (void)c;
    return HB_OK;
}

template <class A, int VARIANT>
int launch_steps(hb_handle *h, hb::DevMesh<typename A::real> &m, int n, cudaStream_t st) {
    const int grid = m.ntiles;
    auto go = [&](auto kern, int threads) {
        for (int k = 0; k < n; k++) kern<<<grid, threads, 0, st>>>(m, k, k == n - 1);
    };
    switch (h->tile_config) {
    case 0: go(hb::step_kernel<A, VARIANT, 256, 2>, 256); break;
    case 1: go(hb::step_kernel<A, VARIANT, 256, 3>, 256); break;
    case 2: go(hb::step_kernel<A, VARIANT, 256, 4>, 256); break;
    case 3: go(hb::step_kernel<A, VARIANT, 128, 6>, 128); break;
    case 4: go(hb::step_kernel<A, VARIANT, 128, 8>, 128); break;
    default: go(hb::step_kernel<A, VARIANT, 512, 2>, 512); break;
    }
    hb::tick_kernel<<<1, 1, 0, st>>>(h->d_ctr, n);
    HB_CUDA_RET(cudaGetLastError());
    return HB_OK;
}

int enqueue_steps(hb_handle *h, int n, cudaStream_t st) {
    if (n <= 0) return HB_OK;
    const bool f = h->opt.variant == HB_VARIANT_F;
    if (h->fp32()) return f ? launch_steps<hb::F32Fast, 1>(h, h->m32, n, st) : launch_steps<hb::F32Fast, 0>(h, h->m32, n, st);
    return f ? launch_steps<hb::F64Exact, 1>(h, h->m64, n, st) : launch_steps<hb::F64Exact, 0>(h, h->m64, n, st);
}

int check_range(hb_handle *h, long long n) {
    const long long limit = (long long)h->ndays * h->per_day;
    if (h->steps_done + n > limit)
        return hb::set_error(HB_E_INVALID, "step %lld..%lld beyond the boundary tables (%d intervals of %d steps)",
                             h->steps_done, h->steps_done + n, h->ndays, h->per_day);
    return HB_OK;
}

}  // namespace

extern "C" int hb_tile_configs(int32_t *threads, int32_t *min_blocks, int32_t capacity) {
    for (int i = 0; i < hb::N_TILE_CONFIGS && i < capacity; i++) {
        if (threads) threads[i] = hb::TILE_CONFIGS[i].threads;
        if (min_blocks) min_blocks[i] = hb::TILE_CONFIGS[i].min_blocks;
    }
    return hb::N_TILE_CONFIGS;
}

extern "C" int hb_create(const hb_mesh_desc *md, const hb_options *opt_in, hb_handle **out) {
    if (!md || !out) return hb::set_error(HB_E_INVALID, "hb_create: null argument");
    *out = nullptr;
    hb_options opt;
    if (opt_in) opt = *opt_in; else hb_options_default(&opt);
    if (opt.precision != HB_FP64 && opt.precision != HB_FP32)
        return hb::set_error(HB_E_INVALID, "hb_create: precision %d not available on this path", opt.precision);
    if (md->cells <= 0 || md->ndays <= 0 || md->steps_per_day < 2 || md->nhq < 0)
        return hb::set_error(HB_E_INVALID, "hb_create: cells=%d ndays=%d steps_per_day=%d", md->cells, md->ndays,
                             md->steps_per_day);
    if (md->cells > (1 << 29)) return hb::set_error(HB_E_TOO_LARGE, "hb_create: %d cells", md->cells);
    const double *need[] = {md->nac, md->klas, md->side, md->cosf, md->sinf, md->zbc, md->area, md->fnc,
                            md->bfeat, md->qt, md->dqt, md->zt, md->dzt};
    for (const double *p : need) if (!p) return hb::set_error(HB_E_INVALID, "hb_create: missing mesh array");
    if (md->nhq > 0 && (!md->zw || !md->qw || !md->nhq1)) return hb::set_error(HB_E_INVALID, "hb_create: missing rating tables");
    HB_CUDA_RET(cudaSetDevice(opt.device));
    auto h = new hb_handle();
    h->opt = opt;
    h->C = md->cells; h->ndays = md->ndays; h->nhq = md->nhq;
    h->steps_per_day = md->steps_per_day; h->per_day = md->steps_per_day - 1;
    h->dt = md->dt; h->hm1 = md->hm1; h->hm2 = md->hm2; h->jl = md->jl;
    if (opt.tile_config < 0 || opt.tile_config > hb::N_TILE_CONFIGS) {
        delete h;
        return hb::set_error(HB_E_INVALID, "hb_create: tile_config %d outside 0..%d", opt.tile_config, hb::N_TILE_CONFIGS);
    }
    h->tile_config = opt.tile_config == 0 ? hb::DEFAULT_TILE_CONFIG : opt.tile_config - 1;
    const int C = h->C;
    // neighbour lists in input order, for the renumbering
    std::vector<int32_t> nbr_old(4 * (size_t)C, -1);
    for (size_t s = 0; s < 4 * (size_t)C; s++) {
        int nc = (int)(md->nac[s] - 1.0);
        if (nc != -1 && (nc < 0 || nc >= C)) {
            delete h;
            return hb::set_error(HB_E_BADMESH, "NAC[%zu] = %g out of range", s, md->nac[s]);
        }
        nbr_old[s] = nc;
    }
    if (opt.renumber) h->perm = hb::rcm_order(C, nbr_old);
    else { h->perm.resize(C); std::iota(h->perm.begin(), h->perm.end(), 0); }
    h->inv.assign(C, -1);
    for (int i = 0; i < C; i++) h->inv[h->perm[i]] = i;
    h->klas_orig.assign(md->klas, md->klas + 4 * (size_t)C);
    int st;
    if ((st = dev_alloc(h, &h->d_err, 1)) != HB_OK || (st = dev_alloc(h, &h->d_ctr, 1)) != HB_OK ||
        (st = dev_upload(h, &h->d_perm, h->perm)) != HB_OK || (st = dev_alloc(h, &h->d_stage, 5 * (size_t)C)) != HB_OK) {
        delete h;
        return st;
    }
    st = h->fp32() ? build_device_mesh<float>(h, md, h->m32) : build_device_mesh<double>(h, md, h->m64);
    if (st != HB_OK) { delete h; return st; }
    *out = h;
    return HB_OK;
}

extern "C" int hb_destroy(hb_handle *h) {
    delete h;
    return HB_OK;
}

namespace {
template <class R>
int set_state_t(hb_handle *h, hb::DevMesh<R> &m, const double *H, const double *U, const double *V, const double *Z,
                const double *W) {
    const int C = h->C;
    const int par = (int)(h->steps_done & 1);
    std::vector<R> buf(C);
    const double *src[5] = {H, U, V, Z, W};
    R *dst[5] = {m.H[par], m.U[par], m.V[par], m.Z[par], m.W};
    for (int k = 0; k < 5; k++) {
        if (!src[k]) { if (k < 4) return hb::set_error(HB_E_INVALID, "hb_set_state: missing array"); continue; }
        for (int i = 0; i < C; i++) buf[i] = (R)src[k][h->perm[i]];
        HB_CUDA_RET(cudaMemcpy(dst[k], buf.data(), C * sizeof(R), cudaMemcpyHostToDevice));
    }
    return HB_OK;
}
template <class R>
int get_state_t(hb_handle *h, hb::DevMesh<R> &m, double *H, double *U, double *V, double *Z, double *W) {
    const int C = h->C;
    const int par = (int)(h->steps_done & 1);
    std::vector<R> buf(C);
    double *dst[5] = {H, U, V, Z, W};
    R *src[5] = {m.H[par], m.U[par], m.V[par], m.Z[par], m.W};
    HB_CUDA_RET(cudaDeviceSynchronize());
    for (int k = 0; k < 5; k++) {
        if (!dst[k]) continue;
        HB_CUDA_RET(cudaMemcpy(buf.data(), src[k], C * sizeof(R), cudaMemcpyDeviceToHost));
        for (int i = 0; i < C; i++) dst[k][h->perm[i]] = (double)buf[i];
    }
    return HB_OK;
}
template <class R>
int get_flux_t(hb_handle *h, hb::DevMesh<R> &m, double *F0, double *F1, double *F2, double *F3) {
    const int C = h->C;
    const size_t S = 4 * (size_t)C;
    std::vector<R> buf(S);
    double *dst[4] = {F0, F1, F2, F3};
    R *src[4] = {m.f0, m.f1, m.f2, m.f3};
    HB_CUDA_RET(cudaDeviceSynchronize());
    for (int k = 0; k < 4; k++) {
        if (!dst[k]) continue;
        HB_CUDA_RET(cudaMemcpy(buf.data(), src[k], S * sizeof(R), cudaMemcpyDeviceToHost));
        for (int i = 0; i < C; i++)
            for (int j = 0; j < 4; j++) dst[k][4 * (size_t)h->perm[i] + j] = (double)buf[4 * (size_t)i + j];
    }
    return HB_OK;
}
template <class R>
int get_klas_t(hb_handle *h, hb::DevMesh<R> &m, double *klas) {
    const int C = h->C;
    const size_t S = 4 * (size_t)C;
    std::vector<uint8_t> meta(std::max(h->nslots, 1));
    HB_CUDA_RET(cudaDeviceSynchronize());
    HB_CUDA_RET(cudaMemcpy(meta.data(), m.meta, h->nslots, cudaMemcpyDeviceToHost));
    for (int i = 0; i < C; i++)
        for (int j = 0; j < 4; j++) {
            const size_t so = 4 * (size_t)h->perm[i] + j;
            const int ci = h->slot_index[4 * (size_t)i + j];
            const int code = ci < 0 ? hb::CODE_ZERO : (meta[ci] & hb::META_CODE);
            double k = h->klas_orig[so];
            if (hb::klas_code(k) == hb::CODE_K7 && code == hb::CODE_ZERO) k = 0.0;   // breached (functors.cu:242)
            klas[so] = k;
        }
    return HB_OK;
}
}  // namespace

extern "C" int hb_set_state(hb_handle *h, const double *H, const double *U, const double *V, const double *Z, const double *W) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    return h->fp32() ? set_state_t(h, h->m32, H, U, V, Z, W) : set_state_t(h, h->m64, H, U, V, Z, W);
}
extern "C" int hb_get_state(hb_handle *h, double *H, double *U, double *V, double *Z, double *W) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    return h->fp32() ? get_state_t(h, h->m32, H, U, V, Z, W) : get_state_t(h, h->m64, H, U, V, Z, W);
}
extern "C" int hb_get_flux(hb_handle *h, double *F0, double *F1, double *F2, double *F3) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    return h->fp32() ? get_flux_t(h, h->m32, F0, F1, F2, F3) : get_flux_t(h, h->m64, F0, F1, F2, F3);
}
extern "C" int hb_get_klas(hb_handle *h, double *klas) {
    if (!h || !klas) return hb::set_error(HB_E_INVALID, "null argument");
    return h->fp32() ? get_klas_t(h, h->m32, klas) : get_klas_t(h, h->m64, klas);
}

extern "C" int hb_step(hb_handle *h, int32_t nsteps, void *stream) {
    if (!h || nsteps < 0) return hb::set_error(HB_E_INVALID, "hb_step: bad argument");
    TRY(check_range(h, nsteps));
    TRY(enqueue_steps(h, nsteps, (cudaStream_t)stream));
    h->steps_done += nsteps;
    return HB_OK;
}

namespace {
template <class R>
int step_host_t(hb_handle *h, hb::DevMesh<R> &m, double *H, double *U, double *V, double *Z, double *W, int n,
                cudaStream_t st) {
    const int C = h->C;
    const size_t b = (size_t)C * sizeof(double);
    double *io[5] = {H, U, V, Z, W};
    for (int k = 0; k < 4; k++) HB_CUDA_RET(cudaMemcpyAsync(h->d_stage + (size_t)k * C, io[k], b, cudaMemcpyHostToDevice, st));
    const int blocks = (C + 255) / 256;
    hb::stage_in_kernel<R><<<blocks, 256, 0, st>>>(C, h->d_perm, h->d_stage, h->d_ctr, m.H[0], m.U[0], m.V[0], m.Z[0],
                                                    m.H[1], m.U[1], m.V[1], m.Z[1]);
    HB_CUDA_RET(cudaGetLastError());
    TRY(enqueue_steps(h, n, st));
    hb::stage_out_kernel<R><<<blocks, 256, 0, st>>>(C, h->d_perm, h->d_stage, h->d_ctr, m.H[0], m.U[0], m.V[0], m.Z[0],
                                                     m.H[1], m.U[1], m.V[1], m.Z[1], m.W);
    HB_CUDA_RET(cudaGetLastError());
    for (int k = 0; k < 5; k++)
        if (io[k]) HB_CUDA_RET(cudaMemcpyAsync(io[k], h->d_stage + (size_t)k * C, b, cudaMemcpyDeviceToHost, st));
    return HB_OK;
}
}  // namespace

extern "C" int hb_step_host(hb_handle *h, double *H, double *U, double *V, double *Z, double *W, int32_t nsteps,
                            void *stream) {
    if (!h || !H || !U || !V || !Z || nsteps < 0) return hb::set_error(HB_E_INVALID, "hb_step_host: bad argument");
    TRY(check_range(h, nsteps));
    cudaStream_t st = (cudaStream_t)stream;
    int r = h->fp32() ? step_host_t(h, h->m32, H, U, V, Z, W, nsteps, st) : step_host_t(h, h->m64, H, U, V, Z, W, nsteps, st);
    if (r == HB_OK) h->steps_done += nsteps;
    return r;
}

extern "C" int hb_sync(hb_handle *h, void *stream) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    HB_CUDA_RET(cudaStreamSynchronize((cudaStream_t)stream));
    uint32_t bits = 0;
    HB_CUDA_RET(cudaMemcpy(&bits, h->d_err, sizeof bits, cudaMemcpyDeviceToHost));
    if (bits & hb::ERRBIT_NONFINITE) return hb::set_error(HB_E_NONFINITE, "a step produced a non-finite state");
    if (bits & hb::ERRBIT_UNDEFINED) return hb::set_error(HB_E_UNDEFINED_REF, "a slot without neighbour reached the mirrored Osher branch");
    if (bits & hb::ERRBIT_TABLE_RANGE) return hb::set_error(HB_E_INVALID, "a step ran beyond the boundary tables");
    return HB_OK;
}

extern "C" int hb_device_errors(hb_handle *h, uint32_t *bits) {
    if (!h || !bits) return hb::set_error(HB_E_INVALID, "null argument");
    HB_CUDA_RET(cudaMemcpy(bits, h->d_err, sizeof *bits, cudaMemcpyDeviceToHost));
    return HB_OK;
}

extern "C" int hb_position(hb_handle *h, int64_t *steps_done, int32_t *kt, int32_t *jt) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    if (steps_done) *steps_done = h->steps_done;
    if (kt) *kt = 1 + (int)(h->steps_done % h->per_day);
    if (jt) *jt = (int)(h->steps_done / h->per_day);
    return HB_OK;
}

extern "C" int hb_set_position(hb_handle *h, int64_t steps_done) {
    if (!h || steps_done < 0) return hb::set_error(HB_E_INVALID, "hb_set_position: bad argument");
    HB_CUDA_RET(cudaDeviceSynchronize());
    // keep the state in place: it sits in buffer (steps_done & 1)
    if ((steps_done & 1) != (h->steps_done & 1)) {
        const size_t bytes = (size_t)h->C * (h->fp32() ? sizeof(float) : sizeof(double));
        const int from = (int)(h->steps_done & 1), to = from ^ 1;
        if (h->fp32()) {
            float **B[4] = {h->m32.H, h->m32.U, h->m32.V, h->m32.Z};
            for (auto b : B) HB_CUDA_RET(cudaMemcpy(b[to], b[from], bytes, cudaMemcpyDeviceToDevice));
        } else {
            double **B[4] = {h->m64.H, h->m64.U, h->m64.V, h->m64.Z};
            for (auto b : B) HB_CUDA_RET(cudaMemcpy(b[to], b[from], bytes, cudaMemcpyDeviceToDevice));
        }
    }
    long long v = steps_done;
    HB_CUDA_RET(cudaMemcpy(h->d_ctr, &v, sizeof v, cudaMemcpyHostToDevice));
    h->steps_done = steps_done;
    return HB_OK;
}

extern "C" int hb_capture_graph(hb_handle *h, int32_t nsteps, void *stream) {
    if (!h || nsteps <= 0) return hb::set_error(HB_E_INVALID, "hb_capture_graph: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    cudaStream_t cap = st;
    bool own = false;
    if (!st) { HB_CUDA_RET(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)); own = true; }
    if (h->graph_exec) { cudaGraphExecDestroy(h->graph_exec); h->graph_exec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
    HB_CUDA_RET(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int st2 = enqueue_steps(h, nsteps, cap);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    if (own) cudaStreamDestroy(cap);
    if (st2 != HB_OK) { if (g) cudaGraphDestroy(g); return st2; }
    if (e != cudaSuccess) return hb::set_error(HB_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    h->graph = g;
    HB_CUDA_RET(cudaGraphInstantiate(&h->graph_exec, g, 0));
    h->graph_steps = nsteps;
    return HB_OK;
}

extern "C" int hb_graph_launch(hb_handle *h, void *stream) {
    if (!h || !h->graph_exec) return hb::set_error(HB_E_INVALID, "hb_graph_launch: no graph captured");
    TRY(check_range(h, h->graph_steps));
    HB_CUDA_RET(cudaGraphLaunch(h->graph_exec, (cudaStream_t)stream));
    h->steps_done += h->graph_steps;
    return HB_OK;
}

extern "C" int hb_device_state(hb_handle *h, void **H, void **U, void **V, void **Z, void **W) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    const int par = (int)(h->steps_done & 1);
    if (h->fp32()) {
        if (H) *H = h->m32.H[par]; if (U) *U = h->m32.U[par]; if (V) *V = h->m32.V[par]; if (Z) *Z = h->m32.Z[par];
        if (W) *W = h->m32.W;
    } else {
        if (H) *H = h->m64.H[par]; if (U) *U = h->m64.U[par]; if (V) *V = h->m64.V[par]; if (Z) *Z = h->m64.Z[par];
        if (W) *W = h->m64.W;
    }
    return HB_OK;
}

extern "C" int hb_get_permutation(hb_handle *h, int32_t *perm) {
    if (!h || !perm) return hb::set_error(HB_E_INVALID, "null argument");
    memcpy(perm, h->perm.data(), h->perm.size() * sizeof(int32_t));
    return HB_OK;
}
