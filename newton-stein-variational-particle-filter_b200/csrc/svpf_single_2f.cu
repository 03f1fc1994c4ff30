// svpf_single_2f.cu -- single-filter two-factor tick kernels, every tile shape.
#include "svpf_single.cuh"

namespace svpf {

cudaError_t launch_single_2f(const SingleArgs& a, int C, int tile, cudaStream_t s) {
    if (C < 1 || C > kMaxCluster || a.n < 1) return cudaErrorInvalidValue;
    if (tick_smem_bytes_2f(a.n, C) > max_dyn_smem()) return cudaErrorInvalidValue;
    switch (tile) {
        case 0: return launch_single_t<1, 8, true>(a, C, s);
        case 1: return launch_single_t<1, 4, true>(a, C, s);
        case 2: return launch_single_t<1, 2, true>(a, C, s);
        case 3: return launch_single_t<1, 1, true>(a, C, s);
        case 4: return launch_single_t<2, 1, true>(a, C, s);
        case 5: return launch_single_t<4, 1, true>(a, C, s);
        default: return launch_single_t<8, 1, true>(a, C, s);
    }
}

}  // namespace svpf
