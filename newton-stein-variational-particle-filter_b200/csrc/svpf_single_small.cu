// svpf_single_small.cu -- single-filter tick kernels for tiles with one row
// per thread (column split S = 8, 4, 2, 1), with the mixture's row maximum
// from a min pass (N <= kScanMaxN) or from sorted prior means, each compiled
// for the production configuration alone and for any configuration.
#include "svpf_single.cuh"

namespace svpf {

template <bool SCAN, bool PROD>
static cudaError_t small_tiles(const SingleArgs& a, int C, int tile, cudaStream_t s) {
    switch (tile) {
        case 0: return launch_single_t<1, 8, false, SCAN, PROD>(a, C, s);
        case 1: return launch_single_t<1, 4, false, SCAN, PROD>(a, C, s);
        case 2: return launch_single_t<1, 2, false, SCAN, PROD>(a, C, s);
        default: return launch_single_t<1, 1, false, SCAN, PROD>(a, C, s);
    }
}

cudaError_t launch_single_small(const SingleArgs& a, int C, int tile, cudaStream_t s) {
    const bool prod = is_production_tick(a.cfg);
    if (a.n <= kScanMaxN) return prod ? small_tiles<true, true>(a, C, tile, s) : small_tiles<true, false>(a, C, tile, s);
    return prod ? small_tiles<false, true>(a, C, tile, s) : small_tiles<false, false>(a, C, tile, s);
}

}  // namespace svpf
