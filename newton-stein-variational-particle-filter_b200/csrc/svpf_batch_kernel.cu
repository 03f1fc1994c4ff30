// svpf_batch_kernel.cu -- the persistent batch tick kernel: a grid of
// resident CTAs pulls filters (largest cost first) from a work counter and runs
// each filter's whole tick in shared memory.  No CTA ever waits on another.
#include "svpf_internal.h"
#include "svpf_tick.cuh"
#include "svpf_tick2f.cuh"

namespace svpf {

// Cooperative copy of a POD struct by 4-byte words.
template <class T>
__device__ __forceinline__ void copy_words(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "word copy");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(dst);
    for (int k = threadIdx.x; k < (int)(sizeof(T) / 4); k += kThreads) d[k] = s[k];
}

// PROD: launched only when every single-factor filter of the batch has the
// production configuration (a.prod), so only its code paths are compiled.
template <bool PROD>
__global__ void __launch_bounds__(kThreads, 2) batch_tick_kernel(const __grid_constant__ BatchArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ Plan pl;
    __shared__ svpf_ctl_t ctl;
    __shared__ svpf_config_t cfg;
    __shared__ SVPFParams prm;
    __shared__ svpf_out_t out;
    __shared__ int s_next;
    const Team team{0, 1};
    for (;;) {
        if (threadIdx.x == 0) s_next = atomicAdd(a.queue, 1);
        __syncthreads();
        const int w = s_next;
        if (w >= a.F) break;
        const int f = a.order[w];
        copy_words(&cfg, &a.cfg[f]);
        copy_words(&prm, &a.prm[f]);
        copy_words(&ctl, &a.ctl[f]);
        __syncthreads();
        if (cfg.use_two_factor) {   // two-factor filters run in batch_tick_2f_kernel
            if (threadIdx.x == 0) a.ctl[f].status = SVPF_ERR_UNSUPPORTED;
            continue;
        }
        const int n = a.n[f];
        const long long off = a.off[f];
        const Smem sm = carve(smem, n, 1, 0, a.heun != 0);
        const FilterIO io{a.h + off, a.hp + off, a.v + off, a.lw + off, n};
        const Noise nz{philox_key(a.seed, f), (uint32_t)ctl.timestep, a.tape_n, a.tape_u,
                       a.slots_n, a.slots_u, a.tape_stride, &pl.flag};
        // request mode: y_t from the request, y_prev from the filter's record
        const float yt = a.req_y ? a.req_y[w] : a.y_t[f];
        const float yp = a.req_y ? ctl.y_prev : a.y_prev[f];
        if (threadIdx.x == 0) pl.have_consts = 0;   // make_plan computes the per-tick constants
        if (!refuse_nonfinite(yt, ctl, out)) {   // a refused tick leaves the filter as it was
            const float ypr = readable_y_prev(yp);
            switch (a.tile[f]) {
                case 1: run_tick<1, 4, false, PROD>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                case 2: run_tick<1, 2, false, PROD>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                case 3: run_tick<1, 1, false, PROD>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                case 4: run_tick<2, 1, false, PROD>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                default: run_tick<4, 1, false, PROD>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
            }
            flag_y_prev(yp, ctl);
        }
        if (a.req_y && threadIdx.x == 0 && isfinite(yt)) ctl.y_prev = yt;   // a refused y_t is not kept
        __syncthreads();
        copy_words(&a.ctl[f], &ctl);
        if (a.out != nullptr) copy_words(&a.out[a.req_y ? w : f], &out);
        __syncthreads();
    }
}

// Two-factor filters (their particle segments hold [fast (n); slow (n)]).
__global__ void __launch_bounds__(kThreads, 2) batch_tick_2f_kernel(const __grid_constant__ BatchArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ Plan pl;
    __shared__ svpf_ctl_t ctl;
    __shared__ svpf_config_t cfg;
    __shared__ SVPFParams prm;
    __shared__ svpf_out_t out;
    __shared__ int s_next;
    const Team team{0, 1};
    for (;;) {
        if (threadIdx.x == 0) s_next = atomicAdd(a.queue, 1);
        __syncthreads();
        const int w = s_next;
        if (w >= a.F) break;
        const int f = a.order[w];
        copy_words(&cfg, &a.cfg[f]);
        copy_words(&prm, &a.prm[f]);
        copy_words(&ctl, &a.ctl[f]);
        __syncthreads();
        const int n = a.n[f];
        const long long off = a.off[f];
        const Smem2 sm = carve_2f(smem, n, 1, 0);
        const FilterIO io{a.h + off, a.hp + off, a.v + off, a.lw + off, n};
        const Noise nz{philox_key(a.seed, f), (uint32_t)ctl.timestep, a.tape_n, a.tape_u,
                       a.slots_n, a.slots_u, a.tape_stride, &pl.flag};
        // request mode: y_t from the request, y_prev from the filter's record
        const float yt = a.req_y ? a.req_y[w] : a.y_t[f];
        const float yp = a.req_y ? ctl.y_prev : a.y_prev[f];
        if (!refuse_nonfinite(yt, ctl, out)) {   // a refused tick leaves the filter as it was
            const float ypr = readable_y_prev(yp);
            switch (a.tile[f]) {
                case 1: run_tick_2f<1, 4>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                case 2: run_tick_2f<1, 2>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                case 3: run_tick_2f<1, 1>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                case 4: run_tick_2f<2, 1>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
                default: run_tick_2f<4, 1>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out); break;
            }
            flag_y_prev(yp, ctl);
        }
        if (a.req_y && threadIdx.x == 0 && isfinite(yt)) ctl.y_prev = yt;   // a refused y_t is not kept
        __syncthreads();
        copy_words(&a.ctl[f], &ctl);
        if (a.out != nullptr) copy_words(&a.out[a.req_y ? w : f], &out);
        __syncthreads();
    }
}

// Two-factor filters on clusters of C CTAs (large N: a filter's tick is
// split over C SMs as in the single-filter kernel, which shortens the longest
// tick of a launch C-fold).  Rank 0 takes the next filter from the work
// counter and writes its index into every member's shared memory; cluster
// barriers separate the rounds, so no member waits on a flag.
template <int C>
__global__ void __launch_bounds__(kThreads) batch_tick_2f_cluster_kernel(const __grid_constant__ BatchArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ Plan pl;
    __shared__ svpf_ctl_t ctl;
    __shared__ svpf_config_t cfg;
    __shared__ SVPFParams prm;
    __shared__ svpf_out_t out;
    __shared__ int s_next;
    cg::cluster_group cl = cg::this_cluster();
    const Team team{(int)cl.block_rank(), C};
    for (;;) {
        if (team.rank == 0 && threadIdx.x == 0) {
            const int w = atomicAdd(a.queue, 1);
            for (int r = 0; r < C; ++r) *cl.map_shared_rank(&s_next, r) = w;
        }
        cl.sync();
        const int w = s_next;
        if (w >= a.F) break;
        const int f = a.order[w];
        copy_words(&cfg, &a.cfg[f]);
        copy_words(&prm, &a.prm[f]);
        copy_words(&ctl, &a.ctl[f]);
        __syncthreads();
        const int n = a.n[f];
        const long long off = a.off[f];
        const Smem2 sm = carve_2f(smem, n, C, team.rank);
        const FilterIO io{a.h + off, a.hp + off, a.v + off, a.lw + off, n};
        const Noise nz{philox_key(a.seed, f), (uint32_t)ctl.timestep, a.tape_n, a.tape_u,
                       a.slots_n, a.slots_u, a.tape_stride, &pl.flag};
        const float yt = a.req_y ? a.req_y[w] : a.y_t[f];
        const float yp = a.req_y ? ctl.y_prev : a.y_prev[f];
        if (!refuse_nonfinite(yt, ctl, out)) {   // every member sees the same y_t
            const float ypr = readable_y_prev(yp);
            if ((n + C - 1) / C <= kThreads) run_tick_2f<1, 1>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out);
            else run_tick_2f<2, 1>(cfg, prm, ctl, yt, ypr, io, nz, sm, pl, team, out);
            flag_y_prev(yp, ctl);
        }
        if (team.rank == 0) {
            if (a.req_y && threadIdx.x == 0 && isfinite(yt)) ctl.y_prev = yt;   // a refused y_t is not kept
            __syncthreads();
            copy_words(&a.ctl[f], &ctl);
            if (a.out != nullptr) copy_words(&a.out[a.req_y ? w : f], &out);
        }
        cl.sync();   // every member is done with this filter before the next index is written
    }
}

constexpr int kCluster2f = kClusterMembers2f;

int batch_cluster_grid_2f(size_t smem_bytes) {
    auto kern = batch_tick_2f_cluster_kernel<kCluster2f>;
    if (configure_kernel((const void*)kern, (int)max_dyn_smem(), true) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kCluster2f, 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kCluster2f;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return 0;
    }
    return clusters * kCluster2f;
}

cudaError_t launch_batch_2f_cluster(const BatchArgs& a, size_t smem_bytes, int grid, cudaStream_t s) {
    if (grid < kCluster2f) return cudaErrorInvalidConfiguration;
    auto kern = batch_tick_2f_cluster_kernel<kCluster2f>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid / kCluster2f * kCluster2f, 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kCluster2f;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, a);
}

int batch_grid_2f(size_t smem_bytes) {
    if (configure_kernel((const void*)batch_tick_2f_kernel, (int)max_dyn_smem(), false) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_tick_2f_kernel, kThreads, smem_bytes);
    if (per_sm < 1) return 0;
    return sms * per_sm;
}

cudaError_t launch_batch_2f(const BatchArgs& a, size_t smem_bytes, int grid, cudaStream_t s) {
    if (grid < 1) return cudaErrorInvalidConfiguration;
    batch_tick_2f_kernel<<<grid, kThreads, smem_bytes, s>>>(a);
    return cudaGetLastError();
}

int batch_grid(size_t smem_bytes) {
    if (configure_kernel((const void*)batch_tick_kernel<false>, (int)max_dyn_smem(), false) != cudaSuccess ||
        configure_kernel((const void*)batch_tick_kernel<true>, (int)max_dyn_smem(), false) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // both variants are bounded to 2 CTAs per SM by their launch bounds
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_tick_kernel<false>, kThreads, smem_bytes);
    if (per_sm < 1) return 0;
    return sms * per_sm;
}

cudaError_t launch_batch(const BatchArgs& a, size_t smem_bytes, int grid, cudaStream_t s) {
    if (grid < 1) return cudaErrorInvalidConfiguration;
    if (a.prod) batch_tick_kernel<true><<<grid, kThreads, smem_bytes, s>>>(a);
    else batch_tick_kernel<false><<<grid, kThreads, smem_bytes, s>>>(a);
    return cudaGetLastError();
}

}  // namespace svpf
