// hb_ref_layout.cu -- CalculateFlux / UpdateCell over the caller's own arrays
// in the reference layout (functors.cu:787-818).  One thread per slot for the
// flux, one per cell for the update, like the reference; the arithmetic is the
// shared physics of hb_physics.cuh.
#include "hb_common.cuh"
#include "hb_physics.cuh"
#include "hydrob200_refview.h"

namespace hb {

__device__ uint32_t g_ref_errors;

template <class R>
struct RefView;
template <>
struct RefView<double> { using type = hb_ref_mesh_view; };
template <>
struct RefView<float> { using type = hb_ref_mesh_view_f32; };

template <class A, int VARIANT>
__global__ void __launch_bounds__(256) ref_flux_kernel(typename RefView<typename A::real>::type m, int kt, int jt) {
    using R = typename A::real;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * m.CELL) return;
    const int pos = idx >> 2;
    const auto &c = m.cells;
    const auto &sd = m.sides;
    SlotIn<R> in;
    in.own = {c.H[pos], c.U[pos], c.V[pos], c.Z[pos], c.ZBC[pos]};
    const int nc = (int)(sd.NAC[idx] - R(1));
    in.has_nb = nc != -1;
    in.own_first = pos < nc;
    if (in.has_nb) in.nb = {c.H[nc], c.U[nc], c.V[nc], c.Z[nc], c.ZBC[nc]};
    else in.nb = {R(0), R(0), R(0), R(0), R(0)};
    in.code = klas_code((double)sd.KLAS[idx]);
    in.cosj = sd.COSF[idx];
    in.sinj = sd.SINF[idx];
    in.side = sd.SIDE[idx];
    StepParams p{(double)m.HM1, (double)m.HM2, (double)m.JL, (double)m.DT, kt, jt};
    auto fetch = [&]() {
        BoundaryIn<R> b;
        const size_t t = (size_t)jt * (size_t)m.CELL + (size_t)pos;
        b.qt = c.QT[t]; b.dqt = c.DQT[t]; b.zt = c.ZT[t]; b.dzt = c.DZT[t];
        b.top = c.BoundaryFeature[pos];
        b.zw = c.ZW + (size_t)pos * (size_t)m.NHQ;
        b.qw = c.QW + (size_t)pos * (size_t)m.NHQ;
        b.nhq1 = c.NHQ1[pos];
        b.nhq = m.NHQ;
        return b;
    };
    const R cl = A::sqrt(A::mul(A::c(9.81), in.own.h));
    SlotOut<R> o;
    flux_slot<A, VARIANT>(in, cl, p, fetch, o);
    if (o.undefined) atomicOr(&g_ref_errors, ERRBIT_UNDEFINED);
    if (o.klas_to_zero) sd.KLAS[idx] = R(0);
    if (o.mask & 1) sd.FLUX0[idx] = o.f[0];
    if (o.mask & 2) sd.FLUX1[idx] = o.f[1];
    if (o.mask & 4) sd.FLUX2[idx] = o.f[2];
    if (o.mask & 8) sd.FLUX3[idx] = o.f[3];
}

template <class A, int VARIANT>
__global__ void __launch_bounds__(256) ref_update_kernel(typename RefView<typename A::real>::type m) {
    using R = typename A::real;
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= m.CELL) return;
    const auto &c = m.cells;
    const auto &sd = m.sides;
    R wh = R(0), wu = R(0), wv = R(0);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int s = 4 * pos + j;
        wsum_add<A>(wh, wu, wv, sd.FLUX0[s], sd.FLUX1[s], sd.FLUX2[s], sd.FLUX3[s], sd.SIDE[s], sd.SLCOS[s], sd.SLSIN[s]);
    }
    CellUpdateIn<R> ci;
    ci.h = c.H[pos]; ci.u = c.U[pos]; ci.v = c.V[pos]; ci.zbc = c.ZBC[pos]; ci.fnc = c.FNC[pos];
    if (VARIANT == 1) {
        // SIDEX: triangle inradius or smaller mid-width of a quad (v0 functors.cu:752-763)
        const R s0 = sd.SIDE[4 * pos], s1 = sd.SIDE[4 * pos + 1], s2 = sd.SIDE[4 * pos + 2], s3 = sd.SIDE[4 * pos + 3];
        if (s3 > R(0)) {
            ci.sidex = A::fmin(A::mul(A::c(0.5), A::add(s0, s2)), A::mul(A::c(0.5), A::add(s1, s3)));
        } else {
            R ss = A::mul(A::c(0.5), A::add(A::add(s0, s1), s2));
            ci.sidex = A::sqrt(A::div(A::mul(A::mul(A::sub(ss, s0), A::sub(ss, s1)), A::sub(ss, s2)), ss));
        }
        ci.dta_or_area = c.AREA[pos];
    } else {
        ci.sidex = R(0);
        ci.dta_or_area = A::div(A::c((double)m.DT), c.AREA[pos]);
    }
    StepParams p{(double)m.HM1, (double)m.HM2, (double)m.JL, (double)m.DT, 0, 0};
    CellUpdateOut<R> o = update_cell<A, VARIANT>(ci, wh, wu, wv, p);
    c.H[pos] = o.h; c.U[pos] = o.u; c.V[pos] = o.v; c.Z[pos] = o.z; c.W[pos] = o.w;
}

template <class A, class View>
static int launch_flux(const View *m, int kt, int jt, int variant, void *stream) {
    if (!m || m->CELL < 0) return set_error(HB_E_INVALID, "hb_ref_calculate_flux: bad mesh view");
    if (m->CELL == 0) return HB_OK;
    if (jt < 0 || jt >= m->NDAYS) return set_error(HB_E_INVALID, "hb_ref_calculate_flux: jt=%d outside [0,%d)", jt, m->NDAYS);
    const long long n = 4LL * m->CELL;
    const int blocks = (int)((n + 255) / 256);
    cudaStream_t st = (cudaStream_t)stream;
    if (variant == HB_VARIANT_F) ref_flux_kernel<A, 1><<<blocks, 256, 0, st>>>(*m, kt, jt);
    else ref_flux_kernel<A, 0><<<blocks, 256, 0, st>>>(*m, kt, jt);
    HB_CUDA_RET(cudaGetLastError());
    return HB_OK;
}

template <class A, class View>
static int launch_update(const View *m, int variant, void *stream) {
    if (!m || m->CELL < 0) return set_error(HB_E_INVALID, "hb_ref_update_cell: bad mesh view");
    if (m->CELL == 0) return HB_OK;
    const int blocks = (m->CELL + 255) / 256;
    cudaStream_t st = (cudaStream_t)stream;
    if (variant == HB_VARIANT_F) ref_update_kernel<A, 1><<<blocks, 256, 0, st>>>(*m);
    else ref_update_kernel<A, 0><<<blocks, 256, 0, st>>>(*m);
    HB_CUDA_RET(cudaGetLastError());
    return HB_OK;
}

}  // namespace hb

extern "C" int hb_ref_calculate_flux(const hb_ref_mesh_view *mesh, int32_t kt, int32_t jt, int32_t variant, void *stream) {
    return hb::launch_flux<hb::F64Exact>(mesh, kt, jt, variant, stream);
}
extern "C" int hb_ref_update_cell(const hb_ref_mesh_view *mesh, int32_t variant, void *stream) {
    return hb::launch_update<hb::F64Exact>(mesh, variant, stream);
}
extern "C" int hb_ref_calculate_flux_f32(const hb_ref_mesh_view_f32 *mesh, int32_t kt, int32_t jt, int32_t variant, void *stream) {
    return hb::launch_flux<hb::F32Fast>(mesh, kt, jt, variant, stream);
}
extern "C" int hb_ref_update_cell_f32(const hb_ref_mesh_view_f32 *mesh, int32_t variant, void *stream) {
    return hb::launch_update<hb::F32Fast>(mesh, variant, stream);
}
extern "C" int hb_ref_take_device_errors(uint32_t *bits) {
    uint32_t v = 0, zero = 0;
    HB_CUDA_RET(cudaMemcpyFromSymbol(&v, hb::g_ref_errors, sizeof v));
    HB_CUDA_RET(cudaMemcpyToSymbol(hb::g_ref_errors, &zero, sizeof zero));
    if (bits) *bits = v;
    return HB_OK;
}

// Reference-signature overloads (functors.cuh:59-65).  The reference exits the
// process on a CUDA error (common.hpp:57-59); these report on stderr instead.
static void report(int st, const char *what) {
    if (st != HB_OK) fprintf(stderr, "hydrob200: %s failed: %s\n", what, hb_last_error_string());
}
void CalculateFlux(const MeshView &mesh, int kt, int jt, CUstream_st *stream) {
    report(hb_ref_calculate_flux(reinterpret_cast<const hb_ref_mesh_view *>(&mesh), kt, jt, HB_VARIANT_H, stream),
           "CalculateFlux");
}
void UpdateCell(const MeshView &mesh, CUstream_st *stream) {
    report(hb_ref_update_cell(reinterpret_cast<const hb_ref_mesh_view *>(&mesh), HB_VARIANT_H, stream), "UpdateCell");
}
void CalculateFlux(const MeshView &mesh, int kt, int jt) {
    CalculateFlux(mesh, kt, jt, nullptr);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) fprintf(stderr, "hydrob200: CalculateFlux: %s\n", cudaGetErrorString(e));
}
void UpdateCell(const MeshView &mesh) {
    UpdateCell(mesh, nullptr);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) fprintf(stderr, "hydrob200: UpdateCell: %s\n", cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// hb_ref_step_static: one step with a fixed, library-owned scratch array
// ---------------------------------------------------------------------------
#include <mutex>

namespace hb {

// [HB_REF_STEP_STATIC_MAX_CELLS * 4 slots][4] = {F0, dWU, dWV, SIDE} per slot.
// Host code must not take this name as a device address: it is a host-side
// stand-in; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_static_terms[(size_t)HB_REF_STEP_STATIC_MAX_CELLS * 16];

constexpr int MAX_DEVICES = 64;
static std::mutex g_static_mu;
static double *g_static_ptr[MAX_DEVICES];

// device address of g_static_terms on the current device (looked up once per device)
static int static_terms_ptr(double **out) {
    int dev = -1;
    HB_CUDA_RET(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return set_error(HB_E_INVALID, "hb_ref_step_static: device %d", dev);
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_terms);
        if (e != cudaSuccess || !p)
            return set_error(HB_E_CUDA, "hb_ref_step_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_static_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_static_ptr[dev];
    return HB_OK;
}

// CalculateFluxKernel's writes (FLUX0..3 by the slot's mask, KLAS on breach)
// plus the slot's terms of the cell sums (functors.cu:733-741) into `terms`.
template <int VARIANT>
__global__ void __launch_bounds__(256) static_flux_kernel(hb_ref_mesh_view m, int kt, int jt, double *terms) {
    using A = F64Exact;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * m.CELL) return;
    const int pos = idx >> 2;
    const auto &c = m.cells;
    const auto &sd = m.sides;
    SlotIn<double> in;
    in.own = {c.H[pos], c.U[pos], c.V[pos], c.Z[pos], c.ZBC[pos]};
    const int nc = (int)(sd.NAC[idx] - 1.0);
    in.has_nb = nc != -1;
    in.own_first = pos < nc;
    if (in.has_nb) in.nb = {c.H[nc], c.U[nc], c.V[nc], c.Z[nc], c.ZBC[nc]};
    else in.nb = {0.0, 0.0, 0.0, 0.0, 0.0};
    in.code = klas_code(sd.KLAS[idx]);
    in.cosj = sd.COSF[idx];
    in.sinj = sd.SINF[idx];
    in.side = sd.SIDE[idx];
    StepParams p{m.HM1, m.HM2, m.JL, m.DT, kt, jt};
    auto fetch = [&]() {
        BoundaryIn<double> b;
        const size_t t = (size_t)jt * (size_t)m.CELL + (size_t)pos;
        b.qt = c.QT[t]; b.dqt = c.DQT[t]; b.zt = c.ZT[t]; b.dzt = c.DZT[t];
        b.top = c.BoundaryFeature[pos];
        b.zw = c.ZW + (size_t)pos * (size_t)m.NHQ;
        b.qw = c.QW + (size_t)pos * (size_t)m.NHQ;
        b.nhq1 = c.NHQ1[pos];
        b.nhq = m.NHQ;
        return b;
    };
    SlotOut<double> o;
    flux_slot<A, VARIANT>(in, A::sqrt(A::mul(9.81, in.own.h)), p, fetch, o);
    if (o.undefined) atomicOr(&g_ref_errors, ERRBIT_UNDEFINED);
    if (o.klas_to_zero) sd.KLAS[idx] = 0.0;
    // fluxes this slot does not write keep their values (functors.cu:525-565)
    if (o.mask & 1) sd.FLUX0[idx] = o.f[0]; else o.f[0] = sd.FLUX0[idx];
    if (o.mask & 2) sd.FLUX1[idx] = o.f[1]; else o.f[1] = sd.FLUX1[idx];
    if (o.mask & 4) sd.FLUX2[idx] = o.f[2]; else o.f[2] = sd.FLUX2[idx];
    if (o.mask & 8) sd.FLUX3[idx] = o.f[3]; else o.f[3] = sd.FLUX3[idx];
    const double fr1 = A::add(o.f[1], o.f[3]);
    const double slcos = sd.SLCOS[idx], slsin = sd.SLSIN[idx];
    double *t = terms + 4 * (size_t)idx;
    t[0] = o.f[0];
    t[1] = A::dot(slcos, fr1, -slsin, o.f[2], M_WU);
    t[2] = A::dot(slsin, fr1, slcos, o.f[2], M_WV);
    t[3] = in.side;
}

// UpdateCellKernel (functors.cu:717-784) with the sums taken from `terms`.
template <int VARIANT>
__global__ void __launch_bounds__(256) static_update_kernel(hb_ref_mesh_view m, const double *terms) {
    using A = F64Exact;
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= m.CELL) return;
    const auto &c = m.cells;
    const auto &sd = m.sides;
    double wh = 0.0, wu = 0.0, wv = 0.0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const double *t = terms + 16 * (size_t)pos + 4 * j;
        wh = A::madd(t[3], t[0], wh, M_WH);
        wu = A::add(wu, t[1]);
        wv = A::add(wv, t[2]);
    }
    CellUpdateIn<double> ci;
    ci.h = c.H[pos]; ci.u = c.U[pos]; ci.v = c.V[pos]; ci.zbc = c.ZBC[pos]; ci.fnc = c.FNC[pos];
    if (VARIANT == 1) {
        const double s0 = sd.SIDE[4 * pos], s1 = sd.SIDE[4 * pos + 1], s2 = sd.SIDE[4 * pos + 2], s3 = sd.SIDE[4 * pos + 3];
        if (s3 > 0.0) {
            ci.sidex = A::fmin(A::mul(0.5, A::add(s0, s2)), A::mul(0.5, A::add(s1, s3)));
        } else {
            double ss = A::mul(0.5, A::add(A::add(s0, s1), s2));
            ci.sidex = A::sqrt(A::div(A::mul(A::mul(A::sub(ss, s0), A::sub(ss, s1)), A::sub(ss, s2)), ss));
        }
        ci.dta_or_area = c.AREA[pos];
    } else {
        ci.sidex = 0.0;
        ci.dta_or_area = A::div(m.DT, c.AREA[pos]);
    }
    StepParams p{m.HM1, m.HM2, m.JL, m.DT, 0, 0};
    CellUpdateOut<double> o = update_cell<A, VARIANT>(ci, wh, wu, wv, p);
    c.H[pos] = o.h; c.U[pos] = o.u; c.V[pos] = o.v; c.Z[pos] = o.z; c.W[pos] = o.w;
}

}  // namespace hb

extern "C" int hb_ref_step_static(const hb_ref_mesh_view *m, int32_t kt, int32_t jt, int32_t variant, void *stream) {
    if (!m || m->CELL < 0) return hb::set_error(HB_E_INVALID, "hb_ref_step_static: bad mesh view");
    if (m->CELL > HB_REF_STEP_STATIC_MAX_CELLS)
        return hb::set_error(HB_E_TOO_LARGE, "hb_ref_step_static: %d cells, the fixed scratch holds %d", m->CELL,
                             HB_REF_STEP_STATIC_MAX_CELLS);
    if (m->CELL == 0) return HB_OK;
    if (jt < 0 || jt >= m->NDAYS)
        return hb::set_error(HB_E_INVALID, "hb_ref_step_static: jt=%d outside [0,%d)", jt, m->NDAYS);
    double *terms = nullptr;
    int st = hb::static_terms_ptr(&terms);
    if (st != HB_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int fb = (4 * m->CELL + 255) / 256, ub = (m->CELL + 255) / 256;
    if (variant == HB_VARIANT_F) {
        hb::static_flux_kernel<1><<<fb, 256, 0, s>>>(*m, kt, jt, terms);
        hb::static_update_kernel<1><<<ub, 256, 0, s>>>(*m, terms);
    } else {
        hb::static_flux_kernel<0><<<fb, 256, 0, s>>>(*m, kt, jt, terms);
        hb::static_update_kernel<0><<<ub, 256, 0, s>>>(*m, terms);
    }
    HB_CUDA_RET(cudaGetLastError());
    return HB_OK;
}
