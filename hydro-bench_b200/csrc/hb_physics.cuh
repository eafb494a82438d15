// hb_physics.cuh -- the per-slot flux and per-cell update of hydro-cal.
//
// Follows cuda_native_impl/hydro-cal-src/src/functors.cu (variant H) and
// cuda_native_impl/baselines/native_cuda_v0/fp64/hydro-cal-src/src/functors.cu
// (variant F); each function cites the lines it follows.
//
// Rounding.  The fp64 policy (F64Exact) evaluates every operation with an
// explicit IEEE intrinsic (__dmul_rn, __dadd_rn, __fma_rn, __ddiv_rn,
// __dsqrt_rn), so the compiler cannot fuse anything on its own.  Where the
// reference build fuses a multiply into an add (nvcc's default -fmad=true),
// the same fusion is written out here: the `mode` arguments of dot() and
// madd() name which product is fused.  The modes were established by
// matching the reference binary's own dumps bit for bit; with them the
// kernels below reproduce the reference's fp64 results exactly no matter
// how they are scheduled or fused into larger kernels.  pow() is CUDA's own.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

namespace hb {

// ---------------------------------------------------------------------------
// constants (common.hpp:44-52, functors.cu)
// ---------------------------------------------------------------------------
struct K {
    static constexpr double C0 = 1.33, C1 = 1.7, VMIN = 0.001, QLUA = 0.0, BRDTH = 100.0;
};

// boundary-code categories; every double KLAS value maps to one of them
// without changing behaviour (functors.cu:109, :151, :532-565)
enum SlotCode : int8_t {
    CODE_ZERO = 0,        // KLAS == 0: interior chain, direct Osher from the lower-numbered side
    CODE_K1 = 1, CODE_K3 = 3, CODE_K4 = 4, CODE_K5 = 5, CODE_K6 = 6, CODE_K7 = 7, CODE_K10 = 10,
    CODE_BOUNDA_OTHER = 2,    // in [1,8] or >= 10 but none of the above: only FLUX2 is written
    CODE_NONZERO_INTERIOR = 9 // not a boundary code and not 0 (e.g. 9, NaN): mirrored Osher
};

__host__ __device__ inline int8_t klas_code(double kp) {
    if ((kp >= 1 && kp <= 8) || kp >= 10) {
        if (kp == 10) return CODE_K10;
        if (kp == 3) return CODE_K3;
        if (kp == 1) return CODE_K1;
        if (kp == 4) return CODE_K4;
        if (kp == 5) return CODE_K5;
        if (kp == 6) return CODE_K6;
        if (kp == 7) return CODE_K7;
        return CODE_BOUNDA_OTHER;
    }
    return kp == 0 ? CODE_ZERO : CODE_NONZERO_INTERIOR;
}
__host__ __device__ inline bool code_is_bounda(int8_t c) { return c != CODE_ZERO && c != CODE_NONZERO_INTERIOR; }

// ---------------------------------------------------------------------------
// arithmetic policies
// ---------------------------------------------------------------------------
// Every policy has a `real` type for the flux/state arithmetic and a `level`
// type for water levels and bed elevations (Z, ZBC, ZT, ZW, crest heights).
// A depth rebuilt from levels (level minus bed) is formed in `level`
// precision and then rounded to `real` (depth()).
struct F64Exact {
    using real = double;
    using level = double;
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    // x / c for a constant c, correctly rounded: RN(x/c) == __ddiv_rn(x, c).
    // Method: Markstein's theorem (P. Markstein, IBM J. Res. Dev. 34(1), 1990;
    // J.-M. Muller et al., Handbook of Floating-Point Arithmetic, ch. 4): if y is
    // within half an ulp of 1/c and q within one ulp of x/c, then
    // RN(q + RN(x - q*c)*y) = RN(x/c), the remainder being exact in an FMA.
    // y = RN(1/c) is folded at compile time; one refinement of q0 = RN(x*y)
    // brings q within one ulp, the second step rounds correctly.  Zeros,
    // infinities, NaNs and |x| outside [2^-900, 2^900] (far from over/underflow
    // of every quotient here) take __ddiv_rn.  Five FP64 operations instead
    // of the ~18 instructions of __ddiv_rn.
    static __device__ __forceinline__ double divk(double x, double c) {
        const double y = 1.0 / c;
        const double ax = ::fabs(x);
        if (ax >= 0x1p-900 && ax <= 0x1p+900) {
            double q = __dmul_rn(x, y);
            double r = __fma_rn(-q, c, x);
            q = __fma_rn(r, y, q);
            r = __fma_rn(-q, c, x);
            return __fma_rn(r, y, q);
        }
        return __ddiv_rn(x, c);
    }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
    static __device__ __forceinline__ double pow(double a, double b) { return ::pow(a, b); }
    static __device__ __forceinline__ double fmax(double a, double b) { return ::fmax(a, b); }
    static __device__ __forceinline__ double fmin(double a, double b) { return ::fmin(a, b); }
    static __device__ __forceinline__ double fabs(double a) { return ::fabs(a); }
    static __device__ __forceinline__ double copysign(double a, double b) { return ::copysign(a, b); }
    static __device__ __forceinline__ double c(double v) { return v; }
    static __device__ __forceinline__ double lc(double v) { return v; }
    static __device__ __forceinline__ double depth(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double lvl(double h) { return h; }
    static __device__ __forceinline__ double ladd(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double lsub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double ldiv(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double lmax(double a, double b) { return ::fmax(a, b); }
    static __device__ __forceinline__ double lmin(double a, double b) { return ::fmin(a, b); }
    static __device__ __forceinline__ double lmadd(double a, double b, double c, int mode) {
        return mode ? __fma_rn(a, b, c) : __dadd_rn(c, __dmul_rn(a, b));
    }
    // a*b + c*d; mode 0 rounds both products, 1 fuses a*b, 2 fuses c*d
    static __device__ __forceinline__ double dot(double a, double b, double c, double d, int mode) {
        return mode == 1 ? __fma_rn(a, b, __dmul_rn(c, d))
             : mode == 2 ? __fma_rn(c, d, __dmul_rn(a, b))
                         : __dadd_rn(__dmul_rn(a, b), __dmul_rn(c, d));
    }
    // c + a*b; mode 0 rounds the product, otherwise fused
    static __device__ __forceinline__ double madd(double a, double b, double c, int mode) {
        return mode ? __fma_rn(a, b, c) : __dadd_rn(c, __dmul_rn(a, b));
    }
};

struct F32Fast {
    using real = float;
    using level = float;
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
    static __device__ __forceinline__ float divk(float x, double c) { return x / (float)c; }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return fmaf(a, b, c); }
    static __device__ __forceinline__ float sqrt(float a) { return sqrtf(a); }
    static __device__ __forceinline__ float pow(float a, float b) { return powf(a, b); }
    static __device__ __forceinline__ float fmax(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float fmin(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fabs(float a) { return fabsf(a); }
    static __device__ __forceinline__ float copysign(float a, float b) { return copysignf(a, b); }
    static __device__ __forceinline__ float c(double v) { return (float)v; }
    static __device__ __forceinline__ float lc(double v) { return (float)v; }
    static __device__ __forceinline__ float depth(float a, float b) { return a - b; }
    static __device__ __forceinline__ float lvl(float h) { return h; }
    static __device__ __forceinline__ float ladd(float a, float b) { return a + b; }
    static __device__ __forceinline__ float lsub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float ldiv(float a, float b) { return a / b; }
    static __device__ __forceinline__ float lmax(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float lmin(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float lmadd(float a, float b, float c, int) { return fmaf(a, b, c); }
    static __device__ __forceinline__ float dot(float a, float b, float c, float d, int) { return fmaf(a, b, c * d); }
    static __device__ __forceinline__ float madd(float a, float b, float c, int) { return fmaf(a, b, c); }
};

// Split precision: fluxes, velocities and the depth itself in fp32; water
// levels and bed elevations in fp64, so that a depth rebuilt as level minus
// bed (shallow water over a high bed) keeps its digits.  The depth update is
// Kahan-compensated (update_cell): the state carries the fp32 depth and its
// fp32 compensation term, and the level of a cell is rebuilt in fp64 from both.
struct F32Split : F32Fast {
    using level = double;
    static __device__ __forceinline__ double lc(double v) { return v; }
    static __device__ __forceinline__ float depth(double a, double b) { return __double2float_rn(a - b); }
    static __device__ __forceinline__ double lvl(float h) { return (double)h; }
    static __device__ __forceinline__ double ladd(double a, double b) { return a + b; }
    static __device__ __forceinline__ double lsub(double a, double b) { return a - b; }
    static __device__ __forceinline__ double ldiv(double a, double b) { return a / b; }
    static __device__ __forceinline__ double lmax(double a, double b) { return ::fmax(a, b); }
    static __device__ __forceinline__ double lmin(double a, double b) { return ::fmin(a, b); }
    static __device__ __forceinline__ double lmadd(double a, double b, double c, int) { return ::fma(a, b, c); }
};
template <class A> struct is_split : std::false_type {};
template <> struct is_split<F32Split> : std::true_type {};

// Water level of a split-precision cell, in fp64: bed + depth + compensation.
// The state keeps no level of its own.  At the dry threshold (h == HM1) the
// update always leaves hlo = 0, so there hlo is free to carry the offset of
// an initial level below bed + HM1 (the reference's dry cells keep Z < ZBC
// while H = HM1, mesh.cpp:350-361); the depth update ignores it.
template <class A>
__device__ __forceinline__ double split_level(float h, float hlo, double zbc) {
    return (double)h + ((double)hlo + zbc);
}

// Fusion modes of the reference sm_100a build (see file comment).
enum : int {
    M_QL1 = 2, M_QL2 = 1, M_UR = 1, M_QR2 = 1,          // functors.cu:90-91, :153, :158
    M_QL1M = 2, M_QL2M = 2, M_UR1 = 2, M_QR2M = 1,      // :176-177, :181, :186
    M_ACC0 = 0, M_ACC123 = 1,                           // Osher sums, :453-497
    M_SHALLOW_VT = 1,                                   // :130
    M_K10 = 1, M_K1 = 1, M_FIAL1 = 1, M_FIAR1 = 1,      // :209, :376, :379, :383
    M_K3Q = 1, M_FIAL3 = 1, M_FIAR3 = 1, M_LAQP = 1,    // :327, :355, :359, :439
    M_K6UN = 1, M_K6VT = 1,                             // :280-281, :293-294
    M_WH = 1, M_WU = 1, M_WV = 2,                       // :739-741
    M_H2 = 1, M_U2A = 1, M_U2B = 1, M_SQ1 = 1, M_SQ2 = 1 // :754, :771-772, :770, :777
};

static_assert(M_QL1 == M_QL1M && M_QR2 == M_QR2M, "flux_slot shares these modes between the two Osher routes");

// ---------------------------------------------------------------------------
// inputs / outputs of one slot
// ---------------------------------------------------------------------------
template <class R, class L = R>
struct CellState { R h, u, v; L z, zbc; };

template <class R, class L = R>
struct SlotIn {
    CellState<R, L> own;    // H1, U1, V1, Z1 and ZBC of the slot's cell
    CellState<R, L> nb;     // raw H, U, V, Z, ZBC of the neighbour (unused when has_nb == false)
    bool has_nb;            // NAC != 0
    bool own_first;         // pos < NC in the reference numbering
    int8_t code;            // klas_code(KLAS)
    R cosj, sinj, side;     // COSF, SINF, SIDE of the slot
};

// boundary tables at (jt, pos), fetched only for boundary slots
template <class R, class L = R>
struct BoundaryIn {
    R qt, dqt;                      // QT, DQT at [jt][pos]
    L zt, dzt, top;                 // ZT, DZT at [jt][pos]; BoundaryFeature[pos]
    const L *zw;                    // rating-curve levels of the cell
    const R *qw;                    // rating-curve discharges of the cell
    int nhq1;                       // points used (NHQ1[pos])
    int nhq;                        // row width (NHQ)
};
template <class A> using CellStateA = CellState<typename A::real, typename A::level>;
template <class A> using SlotInA = SlotIn<typename A::real, typename A::level>;
template <class A> using BoundaryInA = BoundaryIn<typename A::real, typename A::level>;

template <class R>
struct SlotOut {
    R f[4];
    uint8_t mask;        // bit i set: FLUX<i> written this step (otherwise keeps its old value)
    bool klas_to_zero;   // a breach slot opened (functors.cu:242)
    bool undefined;      // reached the reference's read of H[-1] (functors.cu:170)
};

struct StepParams {
    double hm1, hm2, jl, dt;
    int kt, jt;
};

// ---------------------------------------------------------------------------
// Osher approximate Riemann solver, functors.cu:445-511, :570-712
// ---------------------------------------------------------------------------
// out += sign * QF(h, u, v) with the reference build's sums (functors.cu:453-497, :505-511)
template <class A>
__device__ __forceinline__ void qf_acc(typename A::real out[4], typename A::real h, typename A::real u,
                                       typename A::real v, int sign) {
    using R = typename A::real;
    R f0 = A::mul(h, u);
    R sh = sign > 0 ? h : -h;
    R sf0 = sign > 0 ? f0 : -f0;
    out[0] = A::madd(sh, u, out[0], M_ACC0);
    out[1] = A::madd(sf0, u, out[1], M_ACC123);
    out[2] = A::madd(sf0, v, out[2], M_ACC123);
    R h4 = A::mul(A::c(4.905), h);
    out[3] = A::madd(sign > 0 ? h4 : -h4, h, out[3], M_ACC123);
}

// Per-piece record of one Osher evaluation, for re-summing FLUX2 with another
// tangential velocity: f0[i] = h*u of piece i (pieces 1, 2, 3, 5, 6, 7 in that
// order; 1-3 carry QL's tangent, 5-7 QR's), act/neg bit i = added / subtracted.
template <class R>
struct OsherTrace {
    R f0[6];
    unsigned act, neg;
    __device__ __forceinline__ void set(int i, R v) { f0[i] = v; }
    __device__ __forceinline__ R get(int i) const { return f0[i]; }
};
// The same record with the products kept in a store the caller provides
// (TS: set(i, v) / get(i)), e.g. shared memory: they are read back only for
// the rare re-summed FLUX2, so they need not occupy registers across the rest
// of the evaluation.
template <class TS>
struct OsherTraceIn {
    TS *ts;
    unsigned act, neg;
    template <class R> __device__ __forceinline__ void set(int i, R v) { ts->set(i, v); }
    __device__ __forceinline__ auto get(int i) const { return ts->get(i); }
};

// out += QF(h, u, v) (or -=, `neg`) when `on`, with the reference build's sums
// (functors.cu:453-497, :505-511); `out` is untouched otherwise.
template <class A, class TR>
__device__ __forceinline__ void qf_acc_if(typename A::real out[4], bool on, bool neg, typename A::real h,
                                          typename A::real u, typename A::real v, TR *tr, int piece) {
    using R = typename A::real;
    R f0 = A::mul(h, u);
    R sh = neg ? -h : h;
    R sf0 = neg ? -f0 : f0;
    R h4 = A::mul(A::c(4.905), h);
    R o0 = A::madd(sh, u, out[0], M_ACC0);
    R o1 = A::madd(sf0, u, out[1], M_ACC123);
    R o2 = A::madd(sf0, v, out[2], M_ACC123);
    R o3 = A::madd(neg ? -h4 : h4, h, out[3], M_ACC123);
    if (on) { out[0] = o0; out[1] = o1; out[2] = o2; out[3] = o3; }
    if constexpr (!std::is_same<TR, void>::value) {
        tr->set(piece, f0);
        tr->act |= (on ? 1u : 0u) << piece;
        tr->neg |= (neg ? 1u : 0u) << piece;
    }
}

// A piece that is not taken: traced as inactive (osher_f2 skips it).
template <class A, class TR>
__device__ __forceinline__ void qf_skip(TR *tr, int piece) {
    if constexpr (!std::is_same<TR, void>::value) tr->set(piece, typename A::real(0));
}

// FLUX2 of a traced Osher evaluation re-summed with tangents ql2 / qr2, in the
// same order and with the same fused sums as qf_acc_if.
template <class A, class TR>
__device__ __forceinline__ typename A::real osher_f2(const TR &tr, typename A::real ql2, typename A::real qr2) {
    using R = typename A::real;
    R acc = R(0);
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const R v = i < 3 ? ql2 : qr2;
        const R f0 = tr.get(i);
        const R sf0 = ((tr.neg >> i) & 1u) ? -f0 : f0;
        const R o2 = A::madd(sf0, v, acc, M_ACC123);
        if ((tr.act >> i) & 1u) acc = o2;
    }
    return acc;
}

// OSHER(pos, H_pre, QL, QR, FIL, FLR_OSHER), functors.cu:570-712, with the
// sub-integrals QS<1..7> of :445-503.  `cl` is sqrt(9.81*h_left), the value
// the reference recomputes at :577.
//
// The reference's 16 (K1, K2) cases each add a signed subset of the pieces
// 1 (left state), 2 (left sonic point), 3 (intermediate state, left),
// 5 (intermediate state, right), 6 (right sonic point), 7 (right state), and
// every case lists its pieces in increasing order.  Here the six pieces are
// taken in that order and each is added when its case coefficient is
// non-zero: the same sums in the same order, without one branch per case.
// Pieces without a division are formed on every lane and selected; those
// with one are formed only by the lanes that take them.
// Piece 3 updates FIL and piece 5 updates FIR (QS<3>, QS<5>); no case has
// both, and piece 6 sees the FIR that piece 5 left.
template <class A, class TR = void>
__device__ __forceinline__ void osher(typename A::real cl, const typename A::real ql[3],
                                      const typename A::real qr[3], typename A::real fil,
                                      typename A::real out[4], TR *tr = nullptr) {
    using R = typename A::real;
    if constexpr (!std::is_same<TR, void>::value) { tr->act = 0; tr->neg = 0; }
    R cr = A::sqrt(A::mul(A::c(9.81), qr[0]));
    R fir = A::sub(qr[1], A::mul(A::c(2.0), cr));
    R ua = A::mul(A::add(fil, fir), A::c(0.5));
    R ca = A::fabs(A::mul(A::sub(fil, fir), A::c(0.25)));
    out[0] = out[1] = out[2] = out[3] = R(0);
    int k2 = 0, k1 = 0;
    if (ca < ua) k2 = 1;
    else if (ua >= R(0) && ua < ca) k2 = 2;
    else if (ua >= -ca && ua < R(0)) k2 = 3;
    else if (ua < -ca) k2 = 4;
    if (ql[1] < cl && qr[1] >= -cr) k1 = 1;
    else if (ql[1] >= cl && qr[1] >= -cr) k1 = 2;
    else if (ql[1] < cl && qr[1] < -cr) k1 = 3;
    else if (ql[1] >= cl && qr[1] < -cr) k1 = 4;
    const bool any = k1 != 0 && k2 != 0;
    // coefficients of the pieces (functors.cu:612-711)
    const bool p1 = any && (k1 == 2 || k1 == 4);
    const bool p2 = any && (k2 == 1 ? (k1 == 1 || k1 == 3) : (k1 == 2 || k1 == 4));
    const bool n2 = k2 != 1;                                   // piece 2 subtracted
    const bool p3 = any && k2 == 2;
    const bool p5 = any && k2 == 3;
    const bool p6 = any && (k2 == 4 ? k1 <= 2 : k1 >= 3);
    const bool n6 = k2 != 4;                                   // piece 6 subtracted
    const bool p7 = any && k1 >= 3;
    // Every piece is evaluated only where its case takes it: pieces 2, 3, 5
    // and 6 divide, and subcritical flow mostly takes 3 or 5 alone; pieces 1
    // and 7 (supercritical flow out of a side) are rare, so a warp usually
    // skips them altogether.
    // piece 1: QF(QL)
    if (p1) qf_acc_if<A>(out, true, false, ql[0], ql[1], ql[2], tr, 0);
    else qf_skip<A>(tr, 0);
    // piece 2: US = FIL/3, HS = US^2/9.81
    if (p2) {
        R us = A::divk(fil, 3.0);
        R hs = A::divk(A::mul(us, us), 9.81);
        qf_acc_if<A>(out, true, n2, hs, us, ql[2], tr, 1);
    } else {
        qf_skip<A>(tr, 1);
    }
    // pieces 3 and 5 share UA = (FIL + FIR)/2 and the same arithmetic on
    // their own inputs (FIL - UA with QL's tangent, FIR - UA with QR's); no
    // case takes both, so one code path forms whichever is taken and a warp
    // whose lanes take different ones runs it once
    const R ua35 = A::mul(A::add(fil, fir), A::c(0.5));
    const R fir5 = A::sub(fir, ua35);
    if (p3 || p5) {
        const R d = p3 ? A::sub(fil, ua35) : fir5;
        const R ha = A::divk(A::mul(d, d), 39.24);
        const R vt = p3 ? ql[2] : qr[2];
        const R f0 = A::mul(ha, ua35);
        out[0] = A::madd(ha, ua35, out[0], M_ACC0);
        out[1] = A::madd(f0, ua35, out[1], M_ACC123);
        out[2] = A::madd(f0, vt, out[2], M_ACC123);
        out[3] = A::madd(A::mul(A::c(4.905), ha), ha, out[3], M_ACC123);
        if constexpr (!std::is_same<TR, void>::value) {
            tr->set(2, p3 ? f0 : R(0));
            tr->set(3, p5 ? f0 : R(0));
            tr->act |= (p3 ? 4u : 0u) | (p5 ? 8u : 0u);
        }
    } else {
        qf_skip<A>(tr, 2);
        qf_skip<A>(tr, 3);
    }
    // piece 6: US = FIR/3 with FIR as piece 5 left it
    if (p6) {
        R f6 = p5 ? fir5 : fir;
        R us = A::divk(f6, 3.0);
        R hs = A::divk(A::mul(us, us), 9.81);
        qf_acc_if<A>(out, true, n6, hs, us, qr[2], tr, 4);
    } else {
        qf_skip<A>(tr, 4);
    }
    // piece 7: QF(QR)
    if (p7) qf_acc_if<A>(out, true, false, qr[0], qr[1], qr[2], tr, 5);
    else qf_skip<A>(tr, 5);
}

// ---------------------------------------------------------------------------
// boundary slots: BOUNDA and the KLAS branches, functors.cu:204-443, :513-568
// ---------------------------------------------------------------------------
// QD, functors.cu:394-421
template <class A>
__device__ __forceinline__ typename A::real weir_discharge(typename A::level zl, typename A::level zr,
                                                           typename A::level zb) {
    using R = typename A::real;
    using L = typename A::level;
    L zu = A::lmax(zl, zr), zd = A::lmin(zl, zr);
    R h0 = A::depth(zu, zb), hs = A::depth(zd, zb);
    R delta = A::div(hs, h0);
    if (delta <= A::c(0.667)) return A::copysign(A::mul(A::c(0.384), A::pow(h0, A::c(1.5))), A::depth(zl, zr));
    R dh = A::depth(zu, zd);
    if (dh > A::c(0.09)) return A::copysign(A::mul(A::mul(A::c(4.43), hs), A::sqrt(dh)), A::depth(zl, zr));
    return A::copysign(A::divk(A::mul(A::mul(A::mul(A::c(4.43), hs), A::c(0.3)), dh), 0.1), A::depth(zl, zr));
}

// LAQP, functors.cu:423-443: y(x) by linear interpolation in the table (a -> b)
template <class A>
__device__ __forceinline__ void table_lookup(typename A::real x, typename A::level &y, const typename A::real *a,
                                             const typename A::level *b, int ms) {
    if (ms <= 0) return;
    if (x < a[0]) { y = b[0]; return; }
    if (x > a[ms - 1]) { y = b[ms - 1]; return; }
    for (int i = 0; i < ms - 1; i++) {
        if (x >= a[i] && x <= a[i + 1]) {
            y = A::lmadd(A::ldiv(A::lsub(b[i + 1], b[i]), A::lvl(A::sub(a[i + 1], a[i]))), A::lvl(A::sub(x, a[i])),
                         b[i], M_LAQP);
            return;
        }
    }
}

// Arithmetic of the iterated boundary conditions (KLAS 10 depth, KLAS 1 / 3
// Riemann invariant).  Their stopping tests (|change| <= tol) turn a rounding
// difference into a different iteration count and so into a flux difference
// of the order of the tolerance; split precision therefore runs them in fp64
// (a few boundary edges per mesh).  The other policies use their own.
template <class A> struct iter_policy { using type = A; };
template <> struct iter_policy<F32Split> { using type = F64Exact; };
template <class A> using iter_real = typename iter_policy<A>::type::real;

// Riemann-invariant iteration of KLAS 1 / 3 (functors.cu:355-367, :379-391)
template <class A>
__device__ __forceinline__ iter_real<A> invariant_iter(iter_real<A> ql1, iter_real<A> h, iter_real<A> hb1, double tol,
                                                       int mfial, int mfiar) {
    using I = typename iter_policy<A>::type;
    using T = iter_real<A>;
    T fial = I::madd(I::c(6.264), I::sqrt(h), ql1, mfial);
    T ur0 = ql1, urb = ur0;
    T shb = I::sqrt(hb1);
    for (int k = 1; k <= 30; k++) {
        T fiar = I::madd(I::c(-6.264), shb, urb, mfiar);
        T dsum = I::add(fial, fiar), ddif = I::sub(fial, fiar);
        urb = I::divk(I::div(I::mul(I::mul(dsum, ddif), ddif), hb1), 313.92);
        if (I::fabs(I::sub(urb, ur0)) <= I::c(tol)) break;
        ur0 = urb;
    }
    return urb;
}

// Depth at a given-discharge boundary, KLAS 10 (functors.cu:212-224)
template <class A>
__device__ __forceinline__ iter_real<A> inflow_depth(iter_real<A> fil, iter_real<A> f0, iter_real<A> h) {
    using I = typename iter_policy<A>::type;
    using T = iter_real<A>;
    T hb0 = h, hb = T(0);
    for (int k = 1; k <= 20; k++) {
        T w = I::sub(fil, I::div(f0, hb0));
        hb = I::divk(I::mul(w, w), 39.24);
        if (I::fabs(I::sub(hb0, hb)) <= I::c(0.005)) break;
        hb0 = I::add(I::mul(hb0, I::c(0.5)), I::mul(hb, I::c(0.5)));
    }
    return hb;
}

template <class A, int VARIANT, class TableFetch>
__device__ __forceinline__ void bounda(const SlotInA<A> &in, const StepParams &p, typename A::real fil,
                                       typename A::real ql[3], typename A::level zc, typename A::real uc,
                                       typename A::real vc, const TableFetch &fetch, SlotOut<typename A::real> &o) {
    using R = typename A::real;
    using L = typename A::level;
    using I = typename iter_policy<A>::type;
    using T = iter_real<A>;
    const R h = in.own.h;
    const R hm2 = A::c(p.hm2);
    R cl = A::sqrt(A::mul(A::c(9.81), h));
    bool super = (VARIANT == 1) ? (ql[1] > cl) : (ql[1] > cl && h < hm2);
    if (super) {
        o.f[0] = A::mul(h, ql[1]);
        o.f[1] = A::mul(o.f[0], ql[1]);
        o.f[2] = A::mul(o.f[0], ql[2]);
        o.f[3] = A::mul(A::mul(A::c(4.905), h), h);
        o.mask = 0xF;
        return;
    }
    o.f[2] = R(0);
    if (ql[1] > R(0)) o.f[2] = A::mul(A::mul(h, ql[1]), ql[2]);
    o.mask = 0x4;
    switch (in.code) {
    case CODE_K10: {
        BoundaryInA<A> b = fetch();
        R f0 = -A::madd(b.dqt, A::c((double)p.kt), b.qt, M_K10);
        f0 = A::div(f0, in.side);
        const T f0t = (T)f0;
        const T qb2 = I::mul(f0t, f0t);
        const T hb = inflow_depth<A>((T)fil, f0t, (T)h);
        o.f[0] = f0;
        o.f[1] = hb <= T(1) ? R(0) : (R)I::div(qb2, hb);
        o.f[2] = R(0);
        o.f[3] = (R)I::mul(I::mul(I::c(4.905), hb), hb);
        o.mask = 0xF;
        break;
    }
    case CODE_K3: {
        BoundaryInA<A> b = fetch();
        R q3 = A::mul(A::mul(A::dot(in.own.u, in.cosj, in.own.v, in.sinj, M_K3Q), h), in.side);
        q3 = A::fmax(q3, R(0));
        L zq = L(0);   // the reference leaves ZQH1 unset when the cell has no table (NHQ1 = 0)
        table_lookup<A>(q3, zq, b.qw, b.zw, b.nhq1);
        R dzq = A::depth(zq, in.own.z);
        const T hb1 = I::fmax((T)A::lsub(zq, in.own.zbc), I::c(p.hm2));
        R qw1 = b.nhq > 1 ? b.qw[1] : R(0);   // QW_row[1] (functors.cu:347)
        ql[1] = A::fmax(ql[1], R(0));
        if (q3 <= qw1 || hb1 <= I::c(p.hm2) || dzq >= A::c(0.1)) {
            o.f[0] = A::mul(h, ql[1]);
            o.f[1] = A::mul(o.f[0], ql[1]);
            o.f[3] = A::mul(A::mul(A::c(4.905), h), h);
        } else {
            const T urb = invariant_iter<A>((T)ql[1], (T)h, hb1, 0.001, M_FIAL3, M_FIAR3);
            const T f0 = I::mul(hb1, urb);
            o.f[0] = (R)f0;
            o.f[1] = (R)I::mul(f0, urb);
            o.f[3] = (R)I::mul(I::mul(I::c(4.905), hb1), hb1);
        }
        o.mask = 0xF;
        break;
    }
    case CODE_K1: {
        BoundaryInA<A> b = fetch();
        int mult = VARIANT == 1 ? p.kt : p.jt;
        const T hb1 = I::fmax((T)A::lsub(A::lmadd(b.dzt, A::lc((double)mult), b.zt, M_K1), in.own.zbc), I::c(p.hm2));
        const T urb = invariant_iter<A>((T)ql[1], (T)h, hb1, 0.0001, M_FIAL1, M_FIAR1);
        const T f0 = I::mul(hb1, urb);
        o.f[0] = (R)f0;
        o.f[1] = (R)I::mul(f0, urb);
        o.f[3] = (R)I::mul(I::mul(I::c(4.905), hb1), hb1);
        o.mask = 0xF;
        break;
    }
    case CODE_K4:
        o.f[0] = R(0); o.f[1] = R(0); o.f[2] = R(0);
        o.f[3] = A::mul(A::mul(A::c(4.905), h), h);
        o.mask = 0xF;
        break;
    case CODE_K5: {
        ql[1] = A::fmax(ql[1], R(0));
        o.f[0] = A::mul(h, ql[1]);
        o.f[1] = A::mul(o.f[0], ql[1]);
        R omj = A::sub(A::c(1.0), A::c(p.jl));
        o.f[3] = A::mul(A::mul(A::mul(A::mul(A::c(4.905), h), h), omj), omj);
        o.mask = 0xF;
        break;
    }
    case CODE_K6: {   // CalculataKlas6, functors.cu:258-318
        BoundaryInA<A> b = fetch();
        const L top = b.top, zb = in.own.zbc, zp = in.own.z;
        const R cs = in.cosj, sn = in.sinj;
        if (zp <= top && zc <= top) {
            o.f[0] = R(0); o.f[1] = R(0); o.f[2] = R(0);
            o.f[3] = A::mul(A::mul(A::c(4.905), h), h);
        } else if (zp > top && zc <= top) {
            o.f[0] = A::mul(A::c(K::C0), A::pow(A::depth(zp, top), A::c(1.5)));
            o.f[1] = A::mul(o.f[0], ql[1]);
            o.f[2] = A::mul(o.f[0], ql[2]);
            o.f[3] = A::mul(A::c(4.905), A::pow(A::depth(top, zb), A::c(2.0)));
        } else if (zp <= top && zc > top) {
            o.f[0] = A::mul(A::c(-K::C0), A::pow(A::depth(zc, top), A::c(1.5)));
            o.f[1] = A::mul(o.f[0], A::fmin(A::dot(uc, cs, vc, sn, M_K6UN), R(0)));
            o.f[2] = A::mul(o.f[0], A::dot(vc, cs, -uc, sn, M_K6VT));
            o.f[3] = A::mul(A::c(4.905), A::pow(A::depth(zp, zb), A::c(2.0)));
        } else if (zp > top && zc > top) {
            R dz = A::fabs(A::depth(zp, zc));
            if (zp <= zc) {
                R hd = A::depth(zp, top);
                R un = A::fmin(A::dot(uc, cs, vc, sn, M_K6UN), R(0));
                R vt = A::dot(vc, cs, -uc, sn, M_K6VT);
                R sh = A::add(hd, dz);
                R ce = A::fmin(A::c(1.0), A::mul(A::c(1.05), A::pow(A::div(dz, sh), A::c(0.33333))));
                if (zp < zc && un > R(0)) un = R(0);
                o.f[0] = A::copysign(A::mul(A::mul(ce, A::c(K::C1)), A::pow(sh, A::c(1.5))), A::depth(zp, zc));
                o.f[1] = A::mul(o.f[0], A::fabs(un));
                o.f[2] = A::mul(o.f[0], vt);
                o.f[3] = A::mul(A::c(4.905), A::pow(A::depth(top, zb), A::c(2.0)));
            } else {
                R hd = A::depth(zc, top);
                R un = A::fmax(ql[1], R(0));
                R vt = ql[2];
                R sh = A::add(hd, dz);
                R ce = A::fmin(A::c(1.0), A::mul(A::c(1.05), A::pow(A::div(dz, sh), A::c(0.33333))));
                o.f[0] = A::copysign(A::mul(A::mul(ce, A::c(K::C1)), A::pow(sh, A::c(1.5))), A::depth(zp, zc));
                R dzs = A::depth(zp, zc);
                o.f[1] = A::mul(A::mul(dzs, A::fabs(un)), un);
                o.f[2] = A::mul(A::mul(dzs, A::fabs(un)), vt);
                o.f[3] = A::mul(A::c(4.905), A::pow(A::depth(top, zb), A::c(2.0)));
            }
        }
        o.mask = 0xF;
        break;
    }
    case CODE_K7: {   // CalculateKlas7, functors.cu:234-256
        BoundaryInA<A> b = fetch();
        const L top = b.top, zp = in.own.z;
        if (zp > top || zc > top) {
            o.klas_to_zero = true;
            // The reference reads an uninitialised HB here (functors.cu:246-247); the
            // cell's own depth is used instead.
            R hb = h;
            R cq = weir_discharge<A>(zp, zc, top);
            R cb = A::div(A::c(K::BRDTH), in.side);
            o.f[0] = A::mul(cq, cb);
            o.f[1] = A::mul(cb, A::copysign(A::div(A::mul(cq, cq), hb), cq));
            o.f[3] = A::mul(A::mul(A::c(4.905), hb), hb);
        } else {
            o.f[0] = R(0); o.f[1] = R(0); o.f[2] = R(0);
            o.f[3] = A::mul(A::mul(A::c(4.905), h), h);
        }
        o.mask = 0xF;
        break;
    }
    default:   // codes the reference does not handle: only FLUX2 (functors.cu:525-565)
        break;
    }
}

// ---------------------------------------------------------------------------
// CalculateFluxKernel body for one slot, functors.cu:47-202
// `cl_own` is sqrt(9.81*H) of the slot's cell (the caller may compute it once
// per cell; it is bit-identical to the reference's per-slot value).
//
// ZERO_LEN: the slot is a zero-length edge without neighbour (the unused
// fourth slot of a triangle, mesh.cpp:303-306), and only its contribution
// SIDE*F = 0*F to the cell sums is wanted.  pow(x, 1.5) is then replaced by
// |x| (NaN for x < 0): 0*F keeps the same sign and NaN-ness, so the sums are
// unchanged, and the slot costs no pow.
// ---------------------------------------------------------------------------
template <class A, bool ZERO_LEN>
__device__ __forceinline__ typename A::real pow15(typename A::real x) {
    using R = typename A::real;
    if constexpr (ZERO_LEN) return x < R(0) ? A::div(R(0), R(0)) : A::fabs(x);
    else return A::pow(x, A::c(1.5));
}

// The branch chain of CalculateFluxKernel (functors.cu:98-200): either the
// slot's fluxes are final (returns 0, `o` filled) or it needs Osher across the
// edge: 1 = direct (functors.cu:151-164), 2 = mirrored (:165-200).
template <class A, int VARIANT, class TableFetch, bool ZERO_LEN = false>
__device__ __forceinline__ int flux_chain(const SlotInA<A> &in, typename A::real cl_own,
                                          const StepParams &p, const TableFetch &fetch,
                                          SlotOut<typename A::real> &o) {
    using R = typename A::real;
    using L = typename A::level;
    o.mask = 0xF; o.klas_to_zero = false; o.undefined = false;
    const R HM1 = A::c(p.hm1), HM2 = A::c(p.hm2);
    const R h1 = in.own.h, u1 = in.own.u, v1 = in.own.v;
    const L z1 = in.own.z, zbc1 = in.own.zbc;
    const R cs = in.cosj, sn = in.sinj;
    R ql[3];
    ql[0] = h1;
    ql[1] = A::dot(u1, cs, v1, sn, M_QL1);
    ql[2] = A::dot(v1, cs, -u1, sn, M_QL2);
    L zi = A::lmax(z1, A::ladd(zbc1, A::lc(p.hm1)));
    R hc, uc, vc;
    L bc, zc;
    if (!in.has_nb) { hc = R(0); bc = L(0); zc = L(0); uc = R(0); vc = R(0); }
    else {
        hc = A::fmax(in.nb.h, HM1);
        bc = in.nb.zbc;
        zc = A::lmax(bc, in.nb.z);
        uc = in.nb.u;
        vc = in.nb.v;
    }
    if (code_is_bounda(in.code)) {
        R fil = A::add(ql[1], A::mul(A::c(2.0), cl_own));
        bounda<A, VARIANT>(in, p, fil, ql, zc, uc, vc, fetch, o);
    } else if (h1 <= HM1 && hc <= HM1) {
        o.f[0] = R(0); o.f[1] = R(0); o.f[2] = R(0); o.f[3] = R(0);
    } else if (zi <= bc) {
        o.f[0] = A::mul(A::c(-K::C1), pow15<A, ZERO_LEN>(hc));
        o.f[1] = A::mul(A::mul(h1, ql[1]), A::fabs(ql[1]));
        o.f[2] = R(0);
        o.f[3] = A::mul(A::mul(A::c(4.905), h1), h1);
    } else if (zc <= zbc1) {
        o.f[0] = A::mul(A::c(K::C1), pow15<A, ZERO_LEN>(h1));
        R ha = A::mul(h1, A::fabs(ql[1]));
        o.f[1] = A::mul(ha, ql[1]);
        o.f[2] = A::mul(ha, ql[2]);
        o.f[3] = R(0);
    } else if (h1 <= HM2) {
        if (zc > zi) {
            R dh = A::fmax(A::depth(zc, zbc1), HM1);
            R un = A::mul(A::c(-K::C1), A::sqrt(dh));
            o.f[0] = A::mul(dh, un);
            o.f[1] = A::mul(o.f[0], un);
            o.f[2] = A::mul(o.f[0], A::dot(vc, cs, -uc, sn, M_SHALLOW_VT));
            o.f[3] = A::mul(A::mul(A::c(4.905), h1), h1);
        } else {
            o.f[0] = A::mul(A::c(K::C1), pow15<A, ZERO_LEN>(h1));
            o.f[1] = R(0); o.f[2] = R(0);
            o.f[3] = A::mul(A::mul(A::c(4.905), h1), h1);
        }
    } else if (hc <= HM2) {
        if (zi > zc) {
            R dh = A::fmax(A::depth(zi, bc), HM1);
            R un = A::mul(A::c(K::C1), A::sqrt(dh));
            R hc1 = A::depth(zc, zbc1);
            o.f[0] = A::mul(dh, un);
            o.f[1] = A::mul(o.f[0], un);
            o.f[2] = A::mul(o.f[0], ql[2]);
            o.f[3] = A::mul(A::mul(A::c(4.905), hc1), hc1);
        } else {
            o.f[0] = A::mul(A::c(-K::C1), pow15<A, ZERO_LEN>(hc));
            o.f[1] = A::mul(A::mul(h1, ql[1]), ql[1]);
            o.f[2] = R(0);
            o.f[3] = A::mul(A::mul(A::c(4.905), h1), h1);
        }
    } else if (in.code == CODE_ZERO && in.own_first) {
        return 1;
    } else if (!in.has_nb) {
        // the reference reads H[-1] here (functors.cu:170)
        o.undefined = true;
        o.f[0] = R(0); o.f[1] = R(0); o.f[2] = R(0); o.f[3] = R(0);
    } else {
        return 2;
    }
    return 0;
}

// Osher's inputs across an edge.  Left cell L and right cell R, normal (cs, sn)
// pointing from L to R: the direct route at L and the mirrored route at R see
// the same cells and the same normal (the reversed normal of R's slot), and
// differ only in the fused product of two rotations (M_QL2 vs M_QL2M, M_UR vs
// M_UR1).  `mir` selects the mirrored route's fusions.
template <class R>
struct OsherIn { R cl, fil, hcR, ratio, ur; R ql[3], qr[3]; };

template <class A>
__device__ __forceinline__ OsherIn<typename A::real> osher_inputs(const CellStateA<A> &L,
                                                                 const CellStateA<A> &Rc,
                                                                 typename A::real cs, typename A::real sn,
                                                                 typename A::real clL, bool mir, const StepParams &p) {
    using R = typename A::real;
    const R HM1 = A::c(p.hm1), HM2 = A::c(p.hm2);
    OsherIn<R> o;
    o.cl = clL;
    o.ql[0] = L.h;
    o.ql[1] = A::dot(L.u, cs, L.v, sn, M_QL1);                    // M_QL1 == M_QL1M
    o.ql[2] = mir ? A::dot(L.v, cs, -L.u, sn, M_QL2M) : A::dot(L.v, cs, -L.u, sn, M_QL2);
    o.fil = A::add(o.ql[1], A::mul(A::c(2.0), clL));
    o.hcR = A::fmax(Rc.h, HM1);
    const typename A::level zR = A::lmax(Rc.zbc, Rc.z);
    o.qr[0] = A::fmax(A::depth(zR, L.zbc), HM1);
    o.ur = mir ? A::dot(Rc.u, cs, Rc.v, sn, M_UR1) : A::dot(Rc.u, cs, Rc.v, sn, M_UR);
    o.ratio = A::fmin(A::div(o.hcR, o.qr[0]), A::c(1.5));
    o.qr[1] = A::mul(o.ur, o.ratio);
    if (o.hcR <= HM2 || o.qr[0] <= HM2) o.qr[1] = A::copysign(A::c(K::VMIN), o.ur);
    o.qr[2] = A::dot(Rc.v, cs, -Rc.u, sn, M_QR2);                 // M_QR2 == M_QR2M
    return o;
}

// FLUX1's correction term and the two routes' epilogues (functors.cu:162-163, :191-199).
// The term does not depend on Osher's result, so a caller may form it first
// (osher_f1_term) and add it afterwards: the same two roundings.
template <class A>
__device__ __forceinline__ typename A::real osher_f1_term(typename A::real ratio, typename A::real hcR,
                                                          typename A::real ur) {
    return A::mul(A::mul(A::mul(A::mul(A::sub(A::c(1.0), ratio), hcR), ur), ur), A::c(0.5));
}
template <class A>
__device__ __forceinline__ typename A::real osher_f1(typename A::real fo1, typename A::real ratio,
                                                     typename A::real hcR, typename A::real ur) {
    return A::add(fo1, osher_f1_term<A>(ratio, hcR, ur));
}
template <class A>
__device__ __forceinline__ typename A::real mirror_f3(typename A::real fo3, typename A::level zbcL,
                                                      typename A::level zbc_own) {
    using R = typename A::real;
    typename A::level za = A::ladd(A::lvl(A::sqrt(A::divk(fo3, 4.905))), zbcL);
    R hc3 = R(0);
    if (za > zbc_own) hc3 = A::depth(za, zbc_own);
    return A::mul(A::mul(A::c(4.905), hc3), hc3);
}

// CalculateFluxKernel body for one slot, functors.cu:47-202.
// `cl_own` is sqrt(9.81*H) of the slot's cell (the caller may compute it once
// per cell; it is bit-identical to the reference's per-slot value).
template <class A, int VARIANT, class TableFetch, bool ZERO_LEN = false>
__device__ __forceinline__ void flux_slot(const SlotInA<A> &in, typename A::real cl_own,
                                          const StepParams &p, const TableFetch &fetch,
                                          SlotOut<typename A::real> &o) {
    using R = typename A::real;
    const int route = flux_chain<A, VARIANT, TableFetch, ZERO_LEN>(in, cl_own, p, fetch, o);
    if (route == 0) return;
    const bool mir = route == 2;
    const CellStateA<A> &L = mir ? in.nb : in.own;
    const CellStateA<A> &Rc = mir ? in.own : in.nb;
    const R cs = mir ? -in.cosj : in.cosj, sn = mir ? -in.sinj : in.sinj;
    const R clL = mir ? A::sqrt(A::mul(A::c(9.81), in.nb.h)) : cl_own;
    const OsherIn<R> oi = osher_inputs<A>(L, Rc, cs, sn, clL, mir, p);
    R fo[4];
    osher<A>(oi.cl, oi.ql, oi.qr, oi.fil, fo);
    o.f[1] = osher_f1<A>(fo[1], oi.ratio, oi.hcR, oi.ur);
    o.f[2] = fo[2];
    if (!mir) { o.f[0] = fo[0]; o.f[3] = fo[3]; }
    else { o.f[0] = -fo[0]; o.f[3] = mirror_f3<A>(fo[3], in.nb.zbc, in.own.zbc); }
}

// ---------------------------------------------------------------------------
// UpdateCellKernel body, functors.cu:717-784 (variant F: v0 functors.cu:719-803)
// ---------------------------------------------------------------------------
template <class R, class L = R>
struct CellUpdateIn {
    R h, u, v, fnc;
    L zbc;
    R hlo;             // split precision: the depth's compensation term
    R dta_or_area;     // variant H: DT/AREA; variant F: AREA
    R sidex;           // variant F: the CFL length of the cell (v0 functors.cu:752-763)
};
template <class R, class L = R>
struct CellUpdateOut { R h, u, v, w; L z; R hlo; };

// accumulate slot j's contribution (functors.cu:732-742), in slot order
template <class A>
__device__ __forceinline__ void wsum_add(typename A::real &wh, typename A::real &wu, typename A::real &wv,
                                         typename A::real f0, typename A::real f1, typename A::real f2,
                                         typename A::real f3, typename A::real side, typename A::real slcos,
                                         typename A::real slsin) {
    using R = typename A::real;
    R fr1 = A::add(f1, f3);
    R fr2 = f2;
    wh = A::madd(side, f0, wh, M_WH);
    wu = A::add(wu, A::dot(slcos, fr1, -slsin, fr2, M_WU));
    wv = A::add(wv, A::dot(slsin, fr1, slcos, fr2, M_WV));
}

// Coefficients of a wet cell's velocity update for the reverse sweep (COEF):
// U2 = (H U - DTA WU - DTW U) / H2, DTW = DT FNC S / H^0.33333, S = |(U, V)|
// (functors.cu:766-772).  Eight doubles per cell (two 32-byte halves):
//   {DTW, 1/H2, dDTW/dFNC, dDTW/dH, (dDTW/dS)/S (0 when S = 0), 0, 0, 0}.
constexpr int UPDATE_COEF = 8;

// One 256-bit store of four doubles to global memory (32-byte aligned).
__device__ __forceinline__ void st_global_f64x4(double *p, double x, double y, double z, double w) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" :: "l"(p), "d"(x), "d"(y), "d"(z), "d"(w) : "memory");
}

// COEF: also write the cell's update coefficients to `coef` when the cell is
// wet after the step (H2 > HM2; fp64 only).
template <class A, int VARIANT, bool COEF = false>
__device__ __forceinline__ CellUpdateOut<typename A::real, typename A::level>
update_cell(const CellUpdateIn<typename A::real, typename A::level> &c, typename A::real wh, typename A::real wu,
            typename A::real wv, const StepParams &p, double *coef = nullptr) {
    using R = typename A::real;
    const R HM1 = A::c(p.hm1), HM2 = A::c(p.hm2), DT = A::c(p.dt);
    R dta;
    if (VARIANT == 1) {
        R hside = A::fmax(c.h, HM1);
        R dt2 = A::div(c.sidex, A::add(c.u, A::sqrt(A::mul(A::c(9.81), hside))));
        dt2 = A::fmin(DT, dt2);
        dt2 = A::fmax(dt2, A::divk(DT, 10.0));
        dta = A::div(dt2, c.dta_or_area);
    } else {
        dta = c.dta_or_area;
    }
    const R cap = A::c(VARIANT == 1 ? 5.0 : 15.0);
    CellUpdateOut<R, typename A::level> o;
    o.hlo = R(0);
    if constexpr (is_split<A>::value) {
        // H + (-DTA*WH), Kahan-compensated: (h, hlo) carries the depth to ~2x fp32
        // precision.  A cell at the dry threshold has no compensation (its hlo,
        // if any, is the level offset of split_level, not part of the depth).
        const R comp = c.h > HM1 ? c.hlo : R(0);
        const R y = A::madd(-dta, wh, comp, M_H2);
        const R t = c.h + y;
        o.hlo = y - (t - c.h);
        o.h = t;
        if (!(o.h > HM1)) { o.h = HM1; o.hlo = R(0); }
        o.z = split_level<A>(o.h, o.hlo, c.zbc);
    } else {
        o.h = A::fmax(A::add(A::madd(-dta, wh, c.h, M_H2), A::c(K::QLUA)), HM1);
        o.z = A::ladd(A::lvl(o.h), c.zbc);
    }
    if (o.h <= HM1) {
        o.u = R(0); o.v = R(0);
    } else if (o.h <= HM2) {
        o.u = A::copysign(A::fmin(A::c(K::VMIN), A::fabs(c.u)), c.u);
        o.v = A::copysign(A::fmin(A::c(K::VMIN), A::fabs(c.v)), c.v);
    } else {
        const R sq = A::sqrt(A::dot(c.u, c.u, c.v, c.v, M_SQ1));
        const R hp = A::pow(c.h, A::c(0.33333));
        R wsf = A::div(A::mul(c.fnc, sq), hp);
        R dtw = A::mul(DT, wsf);
        R u2 = A::div(A::madd(-dtw, c.u, A::dot(c.h, c.u, -dta, wu, M_U2A), M_U2B), o.h);
        R v2 = A::div(A::madd(-dtw, c.v, A::dot(c.h, c.v, -dta, wv, M_U2A), M_U2B), o.h);
        o.u = A::copysign(A::fmin(A::fabs(u2), cap), u2);
        o.v = A::copysign(A::fmin(A::fabs(v2), cap), v2);
        if constexpr (COEF) {
            static_assert(std::is_same<R, double>::value, "update coefficients are fp64");
            const double ihp = 1.0 / hp;
            st_global_f64x4(coef, dtw, 1.0 / o.h, DT * sq * ihp, DT * c.fnc * sq * (-0.33333) * ihp / c.h);
            st_global_f64x4(coef + 4, sq > 0.0 ? DT * c.fnc * ihp / sq : 0.0, 0.0, 0.0, 0.0);
        }
    }
    o.w = A::sqrt(A::dot(o.u, o.u, o.v, o.v, M_SQ2));
    return o;
}

}  // namespace hb
