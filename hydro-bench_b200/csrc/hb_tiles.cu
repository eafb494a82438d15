// hb_tiles.cu -- launches of the tile layout: one tile_kernel per step over
// the mesh's tiles, at the launch shape the handle holds.  A translation unit
// of its own so the library's kernels compile in parallel.
#include <algorithm>
#include <type_traits>

#include "hb_handle.hpp"

namespace {

size_t tile_smem_bytes(int max_cells, int max_pairs, size_t real_size) {
    return 16 * real_size * (size_t)max_cells + sizeof(int) * (size_t)max_pairs;
}

// Calls f(kernel, threads) with the tile kernel of a tile-layout launch shape.
template <class A, int VARIANT, class F>
int with_tile_kernel(int config, F &&f) {
    using namespace hb;
    switch (config) {
    case 8: return f(tile_kernel<A, VARIANT, 256, 3>, 256);
    case 9: return f(tile_kernel<A, VARIANT, 256, 2>, 256);
    case 10: return f(tile_kernel<A, VARIANT, 128, 6>, 128);
    case 11: return f(tile_kernel<A, VARIANT, 128, 4>, 128);
    case 12: return f(tile_kernel<A, VARIANT, 512, 1>, 512);
    case 13: return f(tile_kernel<A, VARIANT, 256, 4>, 256);
    case 17: return f(tile_kernel<A, VARIANT, 128, 8>, 128);
    case 18: return f(tile_kernel<A, VARIANT, 256, 5>, 256);
    default: return hb::set_error(HB_E_INVALID, "launch shape %d is not a tile-layout shape", config + 1);
    }
}

template <class A, int VARIANT>
int launch_tiles_t(hb_handle *h, hb::DevMesh<A> m, int n, cudaStream_t st) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)std::max(1, m.ntiles));
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.dynamicSmemBytes = tile_smem_bytes(m.max_tile_cells, m.max_tile_pairs, sizeof(typename A::real));
    const int rc = with_tile_kernel<A, VARIANT>(h->launch_config, [&](auto kernel, int threads) -> int {
        cfg.blockDim = dim3(threads);
        for (int k = 0; k < n; k++) HB_CUDA_RET(cudaLaunchKernelEx(&cfg, kernel, m, k, (int)(k == n - 1)));
        return HB_OK;
    });
    if (rc != HB_OK) return rc;
    return hb_launch_tick(h, n, st);
}

// Lets every tile kernel of the handle's policy use the shared memory its
// largest tile needs (beyond the 48 KB default).
template <class A, int VARIANT>
int set_tile_smem(const hb::DevMesh<A> &m) {
    const size_t bytes = tile_smem_bytes(m.max_tile_cells, m.max_tile_pairs, sizeof(typename A::real));
    for (int c = 0; c < hb::N_LAUNCH_CONFIGS; c++) {
        if (hb::LAUNCH_CONFIGS[c].layout != hb::LAYOUT_TILE) continue;
        const int rc = with_tile_kernel<A, VARIANT>(c, [&](auto kernel, int) -> int {
            HB_CUDA_RET(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
            return HB_OK;
        });
        if (rc != HB_OK) return rc;
    }
    return HB_OK;
}

}  // namespace

int hb_tiles_launch(hb_handle *h, int n, cudaStream_t st) {
    const bool f = h->opt.variant == HB_VARIANT_F;
    return h->with_mesh([&](auto &m) {
        using A = typename std::remove_reference<decltype(m)>::type::Policy;
        return f ? launch_tiles_t<A, 1>(h, m, n, st) : launch_tiles_t<A, 0>(h, m, n, st);
    });
}

int hb_tiles_resident(hb_handle *h, int config, int tile_cells, int *per_sm) {
    const bool f = h->opt.variant == HB_VARIANT_F;
    // shared memory of a tile of up to 5/4 tile_cells cells, with as many
    // mirror pairs as its slots could form (an upper bound)
    const int cells = 5 * tile_cells / 4 + 1;
    return h->with_mesh([&](auto &m) -> int {
        using A = typename std::remove_reference<decltype(m)>::type::Policy;
        const size_t bytes = tile_smem_bytes(cells, 2 * cells, sizeof(typename A::real));
        auto query = [&](auto kernel, int threads) -> int {
            HB_CUDA_RET(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
            HB_CUDA_RET(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kernel, threads, bytes));
            return HB_OK;
        };
        return f ? with_tile_kernel<A, 1>(config, query) : with_tile_kernel<A, 0>(config, query);
    });
}

int hb_tiles_set_smem(hb_handle *h) {
    const bool f = h->opt.variant == HB_VARIANT_F;
    return h->with_mesh([&](auto &m) {
        using A = typename std::remove_reference<decltype(m)>::type::Policy;
        return f ? set_tile_smem<A, 1>(m) : set_tile_smem<A, 0>(m);
    });
}
