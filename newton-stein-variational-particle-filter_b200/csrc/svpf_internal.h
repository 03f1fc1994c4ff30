// svpf_internal.h -- launch interface between the C ABI (svpf_capi.cu) and
// the kernels (svpf_kernels.cu).  Host declarations, plus small helpers
// (SVPF_HD) that device code uses too.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "svpf.h"
#include "svpf_math.h"

namespace svpf {

// Tile shapes <rows per thread R, column split S> compiled into the kernels.
struct TileShape { int R, S; };
constexpr int kNumTiles = 7;
constexpr TileShape kTiles[kNumTiles] = {{1, 8}, {1, 4}, {1, 2}, {1, 1}, {2, 1}, {4, 1}, {8, 1}};
// The batch kernel compiles tiles [kBatchTileLo, kBatchTileHi]: at most four
// rows per thread, which keeps its packed accumulators within the 128
// registers a thread may hold at two CTAs per SM.
constexpr int kBatchTileLo = 1;
constexpr int kBatchTileHi = 5;

// The production configuration: full-Newton transport, Gaussian state noise,
// no Heun step (kernels compiled for it alone carry only its code paths).
inline bool is_production_tick(const svpf_config_t& c) {
    return c.use_newton && c.use_full_newton && !c.use_heun && !c.use_student_t_state;
}

struct SingleArgs {
    svpf_config_t cfg;
    SVPFParams prm;
    svpf_ctl_t ctl;
    float y_t, y_prev;
    float* h;
    float* hp;
    float* v;
    float* lw;
    int n;
    unsigned long long seed;
    const float* tape_n;
    const float* tape_u;
    int slots_n, slots_u;
    svpf_ctl_t* ctl_out;   // host-mapped
    svpf_out_t* out;       // host-mapped
    unsigned int* done;    // host-mapped completion word: seq once ctl_out / out are written
    unsigned int seq;
    int host_consts;       // 1: stc and log_y2 below were computed on the host
    float stc;             // Student-t normaliser of cfg.nu
    double log_y2;         // log(y_t^2 + 1e-8) for the EKF guide
};

struct BatchArgs {
    int F;
    const int* order;      // work order (largest cost first)
    int* queue;            // work counter, zero before each launch
    const int* n;
    const long long* off;
    const uint8_t* tile;
    const svpf_config_t* cfg;
    const SVPFParams* prm;
    svpf_ctl_t* ctl;
    float* h;
    float* hp;
    float* v;
    float* lw;
    const float* y_t;
    const float* y_prev;
    svpf_out_t* out;
    unsigned long long seed;
    const float* tape_n;
    const float* tape_u;
    int slots_n, slots_u, tape_stride;
    int heun;              // any filter of the batch uses Heun (shared-memory layout)
    int prod;              // every single-factor filter has the production configuration
    // request mode (request loop): work item w is filter order[w] with
    // y_t = req_y[w], y_prev = that filter's ctl.y_prev (updated to y_t), and
    // its outputs go to out[w].  nullptr: batch mode (y_t[f], y_prev[f], out[f]).
    const float* req_y;
};

struct InitArgs {
    float* h;
    float* hp;
    float* v;
    const long long* off;   // nullptr: single filter at offset 0
    const int* n;           // per filter (or single n in n0)
    int n0;
    int F;
    const float* mu;        // per filter [F] or nullptr (mu0)
    const float* sd;        // per filter [F] or nullptr (sd0)
    float mu0, sd0;
    unsigned long long seed;
    const float* tape0;     // optional initial normals [slots][tape_stride]: slot 0 the
                            // single-factor draw, slots 1 and 2 the fast and slow draws
    int tape_stride;
    // two-factor filters (svpf_init_two_factor_kernel, svpf_two_factor.cu:29-48)
    const uint8_t* tf;      // per filter [F] or nullptr (tf0)
    int tf0;
    const float* sdf;       // stationary sd of the fast / slow factor, per filter or sdf0/sds0
    const float* sds;
    float sdf0, sds0;
    int key_base;           // filter index of block 0 in the Philox key (request loop: the slot)
    float* h2;              // single filter: separate [2n] arrays for the factors; batch:
    float* hp2;             // nullptr (the filter's own segment holds [fast; slow])
    float* v2;
};

// Dynamic shared-memory bytes of a tick kernel for n particles on C CTAs
// (single-factor, and two-factor).
size_t tick_smem_bytes(int n, int C, bool heun);
// The single-filter kernel's: the tick's layout plus the pre-drawn SVLD normals.
size_t tick_smem_bytes_single(int n, int C, bool heun);
size_t tick_smem_bytes_2f(int n, int C);
// Largest dynamic shared memory a CTA may use on the current device.
size_t max_dyn_smem();
// Current device index in [0, kMaxDevices), or -1.
constexpr int kMaxDevices = 64;
int current_device();
// Set a kernel's dynamic shared-memory opt-in (and, if asked, non-portable
// cluster sizes) on the current device, once per (device, kernel); thread safe.
cudaError_t configure_kernel(const void* func, int dyn_smem_bytes, bool nonportable_cluster);
// Dynamic shared memory a kernel may opt into on the current device (the
// device's per-block opt-in limit less the kernel's static shared memory).
size_t kernel_smem_cap(const void* func);
// Loop counts a tick runs are bounded (the Stein budget of one tick over all
// stages at most SVPF_MAX_STEIN_STEPS, annealing stages at most
// SVPF_MAX_ANNEAL_STEPS), so no configuration keeps a kernel running for long.
SVPF_HD inline bool config_loops_ok(const svpf_config_t& c) {
    if (c.use_two_factor) {
        const int na = c.use_annealing ? c.n_anneal_steps : 1;
        return c.n_stein_steps >= 1 && na >= 1 && na <= SVPF_MAX_ANNEAL_STEPS &&
               (long long)na * c.n_stein_steps <= SVPF_MAX_STEIN_STEPS;
    }
    return c.stein_min_steps >= 0 && c.stein_min_steps <= SVPF_MAX_STEIN_STEPS && c.stein_max_steps >= 0 &&
           c.stein_max_steps <= SVPF_MAX_STEIN_STEPS;
}

// Default tile of the single-filter kernel for n particles on C CTAs, and of
// the batch kernel for n particles.
int default_single_tile(int n, int C);
int default_batch_tile(int n);
// Default cluster size of the single-filter kernel for n particles.
int default_cluster(int n);

cudaError_t launch_single(const SingleArgs& a, int C, int tile, cudaStream_t s);
cudaError_t launch_single_small(const SingleArgs& a, int C, int tile, cudaStream_t s);
cudaError_t launch_single_large(const SingleArgs& a, int C, int tile, cudaStream_t s);
cudaError_t launch_single_2f(const SingleArgs& a, int C, int tile, cudaStream_t s);
cudaError_t launch_batch(const BatchArgs& a, size_t smem_bytes, int grid, cudaStream_t s);
cudaError_t launch_batch_2f(const BatchArgs& a, size_t smem_bytes, int grid, cudaStream_t s);
cudaError_t launch_init(const InitArgs& a, cudaStream_t s);
int batch_grid(size_t smem_bytes);
int batch_grid_2f(size_t smem_bytes);
// Two-factor persistent kernel on clusters of kCluster2f (= 4) CTAs per filter.
int batch_cluster_grid_2f(size_t smem_bytes);   // CTAs (a multiple of 4), 0 if it cannot run
cudaError_t launch_batch_2f_cluster(const BatchArgs& a, size_t smem_bytes, int grid, cudaStream_t s);
constexpr int kClusterMembers2f = 4;
cudaError_t debug_philox(uint32_t k0, uint32_t k1, const uint32_t* d_ctr, uint32_t* d_out, int count);

// Process-wide tuner table: tile chosen for a particle count (-1 = none yet).
int tuned_batch_tile(int n);
void set_tuned_batch_tile(int n, int tile);

}  // namespace svpf
