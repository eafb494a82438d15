// hb_handle.hpp -- the handle's host-side state, shared by hb_solver.cu and
// hb_adjoint.cu.
#pragma once
#include <algorithm>
#include <climits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "hb_step.cuh"

// An NVTX range over a host entry point (visible to Nsight tools; free otherwise).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
namespace hb {
// One scenario of a handle, on the host.
struct Scenario {
    int cells = 0, cell0 = 0;           // its cells: device indices [cell0, cell0 + cells)
    int rec0 = 0, npairs = 0, nrecords = 0;   // its records [rec0, rec0 + nrecords), pairs first
    int ndays = 0, steps_per_day = 0, per_day = 0, nhq = 0;
    double dt = 0, hm1 = 0, hm2 = 0, jl = 0;
    std::vector<int32_t> perm;          // perm[new] = old, within the scenario
    std::vector<int32_t> inv;           // inv[old] = new
    std::vector<double> klas_orig;      // [4 cells] reference order
    std::vector<int32_t> slot_index;    // [4 cells] device slot -> record, -1 = zero-length slot
    std::vector<TileDesc> tiles;        // the whole scenario is one tile in the edge layout
    long long step_limit() const { return (long long)ndays * per_day; }
};
}  // namespace hb

struct hb_handle {
    hb_options opt;
    int C = 0;                       // cells of every scenario
    int max_cells = 0;               // cells of the largest scenario
    std::vector<hb::Scenario> scn;
    std::vector<void *> allocs;
    hb::DevMesh<hb::F64Exact> m64{};
    hb::DevMesh<hb::F32Fast> m32{};
    hb::DevMesh<hb::F32Split> ms{};
    uint32_t *d_err = nullptr;
    long long *d_ctr = nullptr;
    int32_t *d_perm = nullptr;       // scenario permutations, concatenated
    double *d_stage = nullptr;       // [5 max_cells] reference-order staging
    int4 *d_fseg[3] = {nullptr, nullptr, nullptr};   // flux segment tables for 64/128/256 threads
    int nfseg[3] = {0, 0, 0};
    int4 *d_useg = nullptr;
    int nuseg = 0;
    long long steps_done = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_steps = 0;
    int launch_config = 0;           // index into LAUNCH_CONFIGS
    // tile layout: the cells per tile in use; with the balanced default
    // (options' tile_cells = 0) also the resident CTAs of the launch shape on
    // the device and the whole waves of them the tiles must fit in
    int tile_cells = 256, tile_slots = 0, tile_waves = 0;
    // persistent handles: the grid-barrier words {arrival count, give-up flag}
    // (both zeroed before each launch), the resident CTAs of the cooperative
    // launch (0 = not yet queried), and the barrier wait bound
    unsigned *d_bar = nullptr;
    int persist_blocks = 0;
    unsigned long long barrier_limit_ns = 1000000000ull;
    unsigned barrier_phantom = 0;
    struct HaloList { int32_t *cells; int32_t n; };
    std::vector<HaloList> halo_lists;   // hb_halo_define: device cell indices (memory in allocs)
    bool segmented() const { return scn.size() > 1; }
    long long step_limit() const {
        long long l = LLONG_MAX;
        for (const auto &s : scn) l = std::min(l, s.step_limit());
        return l;
    }
    // f(mesh) on the device mesh of this handle's precision
    template <class F> int with_mesh(F &&f) {
        switch (opt.precision) {
        case HB_FP32: return f(m32);
        case HB_SPLIT: return f(ms);
        default: return f(m64);
        }
    }
    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
        graph_steps = 0;
    }
    ~hb_handle() {
        drop_graph();
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

}  // namespace

#define TRY(x) do { int st_ = (x); if (st_ != HB_OK) return st_; } while (0)

// the forward step machinery of hb_solver.cu
int hb_enqueue_steps(hb_handle *h, int n, cudaStream_t st);
// n steps of a plain fp64 edge-layout single mesh (hb_steps_take_mesh) at the
// handle's launch shape, from `m`, a copy of the handle's device mesh with the
// adjoint forward's checkpoint and gauge outputs set
bool hb_steps_take_mesh(const hb_handle *h);
int hb_enqueue_steps_mesh(hb_handle *h, const hb::DevMesh<hb::F64Exact> &m, int n, cudaStream_t st);
int hb_check_range(hb_handle *h, long long n);
int hb_launch_tick(hb_handle *h, int n, cudaStream_t st);
// the tile layout (hb_tiles.cu): n steps at the handle's launch shape, and the
// shared-memory attributes of its tile kernels
int hb_tiles_launch(hb_handle *h, int n, cudaStream_t st);
int hb_tiles_set_smem(hb_handle *h);
// CTAs per SM of a tile-layout launch shape with tiles of about tile_cells cells
int hb_tiles_resident(hb_handle *h, int config, int tile_cells, int *per_sm);
// One fp64 edge-layout step t0 + k (the device step counter must hold t0)
// from state `in` to state `out` ([C][4] each), keeping the slots' terms of
// the cell sums in `terms` ([4C][4]) and the update coefficients of the wet
// cells in `coef` ([C][UPDATE_COEF]); the handle's W is overwritten, its
// fluxes only when `write_flux` is set.
int hb_forward_step_into(hb_handle *h, long long t0, int k, const double *in, double *out, double *terms,
                         double *coef, int write_flux, cudaStream_t st);
