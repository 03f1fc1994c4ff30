// svpf_kernels.cu -- initialisation and debug kernels, launch helpers and the
// tile-shape table of the B200 SVPF engine.  The tick kernels themselves:
//
//   single_tick_kernel<R,S>  (svpf_single_*.cu) one filter, one tick, a
//                            cluster of C <= 16 CTAs sharing particles via DSMEM
//   batch_tick_kernel        (svpf_batch_kernel.cu) many filters, one tick, a
//                            persistent grid pulling filters largest-first
#include <cstdio>
#include <mutex>
#include <set>
#include <unordered_map>
#include <utility>

#include "svpf_internal.h"
#include "svpf_tick.cuh"

namespace svpf {

__global__ void init_kernel(const InitArgs a) {
    // one CTA per filter
    const int f = blockIdx.x;
    const int n = a.n ? a.n[f] : a.n0;
    const long long off = a.off ? a.off[f] : 0;
    const float mu = a.mu ? a.mu[f] : a.mu0;
    const float sd = a.sd ? a.sd[f] : a.sd0;
    const bool tf = a.tf ? a.tf[f] != 0 : a.tf0 != 0;
    const uint2 key = philox_key(a.seed, f + a.key_base);
    auto draw = [&](int i, int slot) {
        if (a.tape0 != nullptr) return a.tape0[(size_t)slot * a.tape_stride + i];
        const uint4 r = philox10(key, make_uint4((uint32_t)i, (uint32_t)slot, 0u, 2u));
        return normal_from_bits(r.x, r.y);
    };
    if (!tf || a.h2 != nullptr) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float h = clamp_h(mu + sd * draw(i, 0));
            a.h[off + i] = h;
            a.hp[off + i] = h;
            a.v[off + i] = 0.0f;
        }
    }
    if (tf) {
        const float sdf = a.sdf ? a.sdf[f] : a.sdf0;
        const float sds = a.sds ? a.sds[f] : a.sds0;
        float* H = a.h2 ? a.h2 : a.h + off;
        float* HP = a.h2 ? a.hp2 : a.hp + off;
        float* V = a.h2 ? a.v2 : a.v + off;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float hf = clamp_h(sdf * draw(i, 1));
            const float hs = clamp_h(sds * draw(i, 2));
            H[i] = hf;
            H[n + i] = hs;
            HP[i] = hf;
            HP[n + i] = hs;
            V[i] = 0.0f;
            V[n + i] = 0.0f;
        }
    }
}

__global__ void philox_kernel(uint32_t k0, uint32_t k1, const uint32_t* ctr, uint32_t* out, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint4 r = philox10(make_uint2(k0, k1), make_uint4(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]));
    out[4 * i] = r.x; out[4 * i + 1] = r.y; out[4 * i + 2] = r.z; out[4 * i + 3] = r.w;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
size_t tick_smem_bytes(int n, int C, bool heun) { return (size_t)smem_floats(n, C, heun) * sizeof(float); }
size_t tick_smem_bytes_single(int n, int C, bool heun) {
    return (size_t)(smem_floats(n, C, heun) + pre_floats(n, C)) * sizeof(float);
}
size_t tick_smem_bytes_2f(int n, int C) { return (size_t)smem_floats_2f(n, C) * sizeof(float); }

// ---- per-device facts and kernel attributes --------------------------------
// Function attributes and device limits belong to a device, so every cache
// below is keyed by the current device; one process may drive several GPUs,
// from several host threads.
static std::mutex g_dev_mu;
static size_t g_max_dyn_smem[kMaxDevices] = {};
static std::set<std::pair<int, const void*>> g_configured;

int current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
    return dev;
}

size_t max_dyn_smem() {
    const int dev = current_device();
    if (dev < 0) return 0;
    std::lock_guard<std::mutex> lk(g_dev_mu);
    if (g_max_dyn_smem[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
        const size_t static_bytes = sizeof(Plan) + sizeof(svpf_ctl_t) + sizeof(svpf_config_t) +
                                    sizeof(SVPFParams) + sizeof(svpf_out_t) + 64;
        g_max_dyn_smem[dev] = (size_t)v > static_bytes ? (size_t)v - static_bytes : 0;
    }
    return g_max_dyn_smem[dev];
}

size_t kernel_smem_cap(const void* func) {
    const int dev = current_device();
    int v = 0;
    cudaFuncAttributes fa{};
    if (dev < 0 || cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, func) != cudaSuccess)
        return 0;
    return (size_t)v > fa.sharedSizeBytes ? (size_t)v - fa.sharedSizeBytes : 0;
}

cudaError_t configure_kernel(const void* func, int dyn_smem_bytes, bool nonportable_cluster) {
    const int dev = current_device();
    if (dev < 0) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_dev_mu);
    if (g_configured.count({dev, func})) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem_bytes);
    if (e == cudaSuccess && nonportable_cluster)
        e = cudaFuncSetAttribute(func, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    g_configured.insert({dev, func});
    return cudaSuccess;
}

int default_cluster(int n) {
    int C = 1;
    while (C < kMaxCluster && n / (2 * C) >= 32) C <<= 1;
    return C;
}

static int rows_per_sweep(int tile) { return kTiles[tile].R * (kThreads / kTiles[tile].S); }

int default_single_tile(int n, int C) {
    const int L = (n + C - 1) / C;
    for (int t = 0; t < kNumTiles; ++t)
        if (rows_per_sweep(t) >= L) return t;
    return kNumTiles - 1;
}

int default_batch_tile(int n) {
    for (int t = kBatchTileLo; t <= kBatchTileHi; ++t)
        if (rows_per_sweep(t) >= n) return t;
    return kBatchTileHi;
}

cudaError_t launch_single(const SingleArgs& a, int C, int tile, cudaStream_t s) {
    if (C < 1 || C > kMaxCluster || a.n < 1) return cudaErrorInvalidValue;
    if (tick_smem_bytes_single(a.n, C, a.cfg.use_heun != 0) > max_dyn_smem()) return cudaErrorInvalidValue;
    return tile <= 3 ? launch_single_small(a, C, tile, s) : launch_single_large(a, C, tile, s);
}

cudaError_t launch_init(const InitArgs& a, cudaStream_t s) {
    if (a.F < 1) return cudaErrorInvalidValue;
    init_kernel<<<a.F, kThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t debug_philox(uint32_t k0, uint32_t k1, const uint32_t* d_ctr, uint32_t* d_out, int count) {
    if (count <= 0) return cudaSuccess;
    philox_kernel<<<(count + 255) / 256, 256>>>(k0, k1, d_ctr, d_out, count);
    return cudaGetLastError();
}

static std::mutex g_tune_mu;
static std::unordered_map<int, int> g_tune;

int tuned_batch_tile(int n) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(n);
    return it == g_tune.end() ? -1 : it->second;
}

void set_tuned_batch_tile(int n, int tile) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[n] = tile;
}

}  // namespace svpf
