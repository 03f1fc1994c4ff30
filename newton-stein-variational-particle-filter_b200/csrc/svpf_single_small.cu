// svpf_single_small.cu -- single-filter tick kernels for tiles with one row
// per thread (column split S = 8, 4, 2, 1), with the mixture's row maximum
// from a min pass (N <= kScanMaxN) or from sorted prior means.
#include "svpf_single.cuh"

namespace svpf {

cudaError_t launch_single_small(const SingleArgs& a, int C, int tile, cudaStream_t s) {
    if (a.n <= kScanMaxN) {
        switch (tile) {
            case 0: return launch_single_t<1, 8, false, true>(a, C, s);
            case 1: return launch_single_t<1, 4, false, true>(a, C, s);
            case 2: return launch_single_t<1, 2, false, true>(a, C, s);
            default: return launch_single_t<1, 1, false, true>(a, C, s);
        }
    }
    switch (tile) {
        case 0: return launch_single_t<1, 8>(a, C, s);
        case 1: return launch_single_t<1, 4>(a, C, s);
        case 2: return launch_single_t<1, 2>(a, C, s);
        default: return launch_single_t<1, 1>(a, C, s);
    }
}

}  // namespace svpf
