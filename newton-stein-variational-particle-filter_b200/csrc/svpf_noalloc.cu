// svpf_noalloc.cu -- a batch tick that allocates nothing.
//
// Some callers cannot call cudaMalloc: a host application that reserves all
// device memory for its own arena at start-up and forbids any allocation
// afterwards, a plugin running inside another framework's memory manager, or
// a latency-critical loop that must not take the implicit device
// synchronisation an allocation can cause.  svpf_batch_tick_noalloc serves
// them: the caller owns and passes every input and output buffer, and the
// kernel's scratch (its work counter, the largest-first work order and the tile
// shape per filter) lives in the file-scope array below, which every GPU that
// loads the library holds until the process exits.
#include <cstring>
#include <mutex>

#include "svpf.h"
#include "svpf_device.cuh"
#include "svpf_internal.h"
#include "svpf_trace.h"

namespace svpf {
namespace {

// Scratch layout, in 4-byte words:
//   [0]                                  work counter
//   [kOrderOff, kOrderOff + kMax)        work order (filter indices)
//   [kTileOff, kTileOff + kMax / 4)      tile shape per filter, one byte each
constexpr int kMax = SVPF_NOALLOC_MAX_FILTERS;
constexpr int kOrderOff = 64;
constexpr int kTileOff = kOrderOff + kMax;
constexpr int kScratchWords = kTileOff + kMax / 4;
constexpr int kBuckets = 14;   // particle counts grouped by bit length (n <= 8192)
static_assert(kBatchTileLo >= 1, "tile 0 marks a filter the setup left out");

static __device__ __align__(256) int g_noalloc_scratch[kScratchWords];

// Device copy of default_batch_tile(): the smallest batch tile whose one sweep
// covers all n rows, else the largest.
__device__ int tile_for(int n) {
    const int rows[kNumTiles] = {kTiles[0].R * (kThreads / kTiles[0].S), kTiles[1].R * (kThreads / kTiles[1].S),
                                 kTiles[2].R * (kThreads / kTiles[2].S), kTiles[3].R * (kThreads / kTiles[3].S),
                                 kTiles[4].R * (kThreads / kTiles[4].S), kTiles[5].R * (kThreads / kTiles[5].S),
                                 kTiles[6].R * (kThreads / kTiles[6].S)};
    for (int t = kBatchTileLo; t <= kBatchTileHi; ++t)
        if (rows[t] >= n) return t;
    return kBatchTileHi;
}

__device__ int bucket_of(int n) {
    int b = 0;
    while ((1 << b) < n && b < kBuckets - 1) ++b;
    return b;
}

// One CTA, before the tick: check every filter against what the launch was
// sized for, choose tiles, and order the valid filters largest first
// (bucketed by particle count; the order inside a bucket is free because the
// filters are independent).  A filter with n outside [1, n_max], an offset
// that is negative or not a multiple of 16 floats, Heun while any_heun is 0,
// or loop counts beyond the engine's limits gets SVPF_ERR_INVALID_ARG in its
// control record (two-factor filters SVPF_ERR_UNSUPPORTED) and is never
// touched by the tick: rejected filters take the first positions of the work
// order and the work counter starts past them.  Every call rewrites all the
// scratch it uses.
__global__ void noalloc_setup_kernel(int F, const int* __restrict__ n, const long long* __restrict__ off,
                                     const svpf_config_t* __restrict__ cfg, svpf_ctl_t* ctl, int n_max,
                                     int any_heun) {
    __shared__ int hist[kBuckets];
    __shared__ int start[kBuckets];
    __shared__ int n_bad, bad_pos;
    int* scratch = g_noalloc_scratch;
    uint8_t* tiles = reinterpret_cast<uint8_t*>(scratch + kTileOff);
    if (threadIdx.x < kBuckets) hist[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        n_bad = 0;
        bad_pos = 0;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < F; f += blockDim.x) {
        const int nf = n[f];
        const long long of = off[f];
        const svpf_config_t& c = cfg[f];
        int st = SVPF_OK;
        if (c.use_two_factor) st = SVPF_ERR_UNSUPPORTED;
        else if (nf < 1 || nf > n_max || of < 0 || (of & 15) != 0 || (c.use_heun && !any_heun) ||
                 !config_loops_ok(c))
            st = SVPF_ERR_INVALID_ARG;
        if (st != SVPF_OK) {
            ctl[f].status = st;
            tiles[f] = 0;   // no batch tile is 0: marks the filter as left out
            atomicAdd(&n_bad, 1);
        } else {
            tiles[f] = (uint8_t)tile_for(nf);
            atomicAdd(&hist[bucket_of(nf)], 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = n_bad;
        for (int b = kBuckets - 1; b >= 0; --b) {   // largest bucket first
            start[b] = acc;
            acc += hist[b];
        }
        scratch[0] = n_bad;   // the work counter starts past the rejected filters
    }
    __syncthreads();
    for (int f = threadIdx.x; f < F; f += blockDim.x) {
        const int pos = tiles[f] == 0 ? atomicAdd(&bad_pos, 1) : atomicAdd(&start[bucket_of(n[f])], 1);
        scratch[kOrderOff + pos] = f;
    }
}

std::mutex g_mu;
int* g_scratch_ptr[256] = {};

// Device address of the scratch array for the current device, looked up once
// per device with that device current.
int* scratch_for_current_device(int* err) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        *err = SVPF_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_scratch_ptr[dev] == nullptr) {
        int* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr) {
            *err = SVPF_ERR_CUDA;
            return nullptr;
        }
        g_scratch_ptr[dev] = ptr;
    }
    return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace svpf

using namespace svpf;

extern "C" {

int svpf_batch_tick_noalloc(int n_filters, const int* d_n, const long long* d_off, const svpf_config_t* d_cfg,
                            const SVPFParams* d_params, svpf_ctl_t* d_ctl, float* d_h, float* d_h_prev,
                            float* d_v, float* d_log_w, const float* d_y_t, const float* d_y_prev,
                            svpf_out_t* d_out, int n_max, int any_heun, unsigned long long seed,
                            cudaStream_t stream) {
    SVPF_TRACE();
    if (n_filters < 1 || n_filters > SVPF_NOALLOC_MAX_FILTERS) return SVPF_ERR_INVALID_ARG;
    if (n_max < 1 || n_max > SVPF_MAX_PARTICLES) return SVPF_ERR_INVALID_ARG;
    if (!d_n || !d_off || !d_cfg || !d_params || !d_ctl || !d_h || !d_h_prev || !d_v || !d_log_w || !d_y_t ||
        !d_y_prev)
        return SVPF_ERR_INVALID_ARG;
    const size_t smem = tick_smem_bytes(n_max, 1, any_heun != 0);
    if (smem > max_dyn_smem()) return SVPF_ERR_INVALID_ARG;
    int err = SVPF_OK;
    int* scratch = scratch_for_current_device(&err);
    if (!scratch) return err;
    const int grid = batch_grid(smem);
    if (grid < 1) return SVPF_ERR_CUDA;
    noalloc_setup_kernel<<<1, kThreads, 0, stream>>>(n_filters, d_n, d_off, d_cfg, d_ctl, n_max, any_heun != 0);
    if (cudaGetLastError() != cudaSuccess) return SVPF_ERR_CUDA;
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.F = n_filters;
    a.order = scratch + kOrderOff;
    a.queue = scratch;
    a.n = d_n;
    a.off = d_off;
    a.tile = reinterpret_cast<const uint8_t*>(scratch + kTileOff);
    a.cfg = d_cfg;
    a.prm = d_params;
    a.ctl = d_ctl;
    a.h = d_h;
    a.hp = d_h_prev;
    a.v = d_v;
    a.lw = d_log_w;
    a.y_t = d_y_t;
    a.y_prev = d_y_prev;
    a.out = d_out;
    a.seed = seed;
    a.tape_stride = n_max;
    a.heun = any_heun != 0;
    return launch_batch(a, smem, grid, stream) == cudaSuccess ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_noalloc_max_filters(void) { return SVPF_NOALLOC_MAX_FILTERS; }

}  // extern "C"
