// svpf_single_large.cu -- single-filter tick kernels for tiles with several
// rows per thread (R = 2, 4, 8; no column split).
#include "svpf_single.cuh"

namespace svpf {

cudaError_t launch_single_large(const SingleArgs& a, int C, int tile, cudaStream_t s) {
    switch (tile) {
        case 4: return launch_single_t<2, 1>(a, C, s);
        case 5: return launch_single_t<4, 1>(a, C, s);
        default: return launch_single_t<8, 1>(a, C, s);
    }
}

}  // namespace svpf
