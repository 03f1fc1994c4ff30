// svpf_single.cuh -- the single-filter tick kernel template (one cluster of
// C <= 16 CTAs per tick) and its launcher; instantiated per tile shape in
// svpf_single_small.cu / svpf_single_large.cu.
#pragma once

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

// The host polls a.done instead of synchronising the stream: the result
// records are made visible system-wide before the sequence number is.
__device__ __forceinline__ void publish_done(const SingleArgs& a) {
    if (a.done) {
        __threadfence_system();
        *reinterpret_cast<volatile unsigned int*>(a.done) = a.seq;
    }
}

template <int R, int S, bool SCAN, bool PROD>
__global__ void __launch_bounds__(kThreads, 1) single_tick_kernel(const __grid_constant__ SingleArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ Plan pl;
    __shared__ svpf_ctl_t ctl;
    __shared__ svpf_config_t cfg;
    __shared__ SVPFParams prm;
    __shared__ svpf_out_t out;
    cg::cluster_group cl = cg::this_cluster();
    const Team team{(int)cl.block_rank(), (int)cl.num_blocks()};
    copy_words(&ctl, &a.ctl);
    copy_words(&cfg, &a.cfg);
    copy_words(&prm, &a.prm);
    __syncthreads();
    Smem sm = carve(smem, a.n, team.size, team.rank, a.cfg.use_heun != 0);
    if (pre_floats(a.n, team.size) > 0) sm.pre = smem + smem_floats(a.n, team.size, a.cfg.use_heun != 0);
    const Noise nz{philox_key(a.seed, 0), (uint32_t)ctl.timestep, a.tape_n, a.tape_u,
                   a.slots_n, a.slots_u, a.n, &pl.flag};
    const FilterIO io{a.h, a.hp, a.v, a.lw, a.n};
    if (threadIdx.x == 0) {
        pl.have_consts = a.host_consts;
        pl.stc = a.stc;
        pl.log_y2 = a.log_y2;
    }
    if (!refuse_nonfinite(a.y_t, ctl, out)) {   // every member sees the same y_t
        run_tick<R, S, SCAN, PROD, kClusterUnroll>(cfg, prm, ctl, a.y_t, readable_y_prev(a.y_prev), io, nz, sm, pl,
                                                   team, out);
        flag_y_prev(a.y_prev, ctl);
    }
    if (team.rank == 0) {
        __syncthreads();
        if (threadIdx.x == 0) {
            *a.ctl_out = ctl;
            *a.out = out;
            publish_done(a);
        }
    }
}

// Two-factor tick: a.h / a.hp / a.v hold [fast (n); slow (n)].
template <int R, int S>
__global__ void __launch_bounds__(kThreads, 1) single_tick_2f_kernel(const __grid_constant__ SingleArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ Plan pl;
    __shared__ svpf_ctl_t ctl;
    __shared__ svpf_config_t cfg;
    __shared__ SVPFParams prm;
    __shared__ svpf_out_t out;
    cg::cluster_group cl = cg::this_cluster();
    const Team team{(int)cl.block_rank(), (int)cl.num_blocks()};
    copy_words(&ctl, &a.ctl);
    copy_words(&cfg, &a.cfg);
    copy_words(&prm, &a.prm);
    __syncthreads();
    const Smem2 sm = carve_2f(smem, a.n, team.size, team.rank);
    const Noise nz{philox_key(a.seed, 0), (uint32_t)ctl.timestep, a.tape_n, a.tape_u,
                   a.slots_n, a.slots_u, a.n, &pl.flag};
    const FilterIO io{a.h, a.hp, a.v, a.lw, a.n};
    if (!refuse_nonfinite(a.y_t, ctl, out)) {   // every member sees the same y_t
        run_tick_2f<R, S>(cfg, prm, ctl, a.y_t, readable_y_prev(a.y_prev), io, nz, sm, pl, team, out);
        flag_y_prev(a.y_prev, ctl);
    }
    if (team.rank == 0) {
        __syncthreads();
        if (threadIdx.x == 0) {
            *a.ctl_out = ctl;
            *a.out = out;
            publish_done(a);
        }
    }
}

// Mixture row maximum of the single-factor tick from a min pass up to this many
// particles (no sort: measured faster on B200 at N <= 1024), from the sorted
// prior means above it.
constexpr int kScanMaxN = 1024;

template <int R, int S, bool TWO_FACTOR = false, bool SCAN = false, bool PROD = false>
static cudaError_t launch_single_t(const SingleArgs& a, int C, cudaStream_t s) {
    const size_t smem = TWO_FACTOR ? tick_smem_bytes_2f(a.n, C) : tick_smem_bytes_single(a.n, C, a.cfg.use_heun != 0);
    auto kern = TWO_FACTOR ? single_tick_2f_kernel<R, S> : single_tick_kernel<R, S, SCAN, PROD>;
    const cudaError_t e = configure_kernel((const void*)kern, (int)max_dyn_smem(), true);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, a);
}

}  // namespace svpf
