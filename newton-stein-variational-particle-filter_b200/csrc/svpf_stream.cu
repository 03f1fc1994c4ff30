// svpf_stream.cu -- request loop over a fleet of instruments (filters) whose
// states live in a fixed HBM budget.
//
// Admission: an instrument's particle state (h, h_prev, v, log_w; 2N floats
// each for a two-factor filter, N otherwise, rounded to 16) is placed
// first-fit in one pool allocated once at creation; an instrument whose state
// does not fit the remaining budget is refused (SVPF_ERR_BUDGET), eviction
// returns its segment to the pool.  No device allocation happens after
// creation.
//
// Requests: a call carries (instrument, y_t) pairs.  Each instrument keeps its
// own y_prev in its control record on the device.  The requests of a call are
// served in rounds -- round r holds the r-th request of every instrument
// named in the call, so one instrument's ticks stay in arrival order -- and
// each round is one persistent launch per model (single-factor,
// two-factor) that pulls its work, largest cost first, from a device list.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <vector>

#include "svpf.h"
#include "svpf_device.cuh"
#include "svpf_internal.h"
#include "svpf_trace.h"

using namespace svpf;

struct svpf_stream {
    int cap = 0;                  // instrument slots
    int n_max = 0;
    size_t budget = 0, pool_floats = 0, fixed_bytes = 0, used_floats = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t side[2] = {nullptr, nullptr};   // the round's two-factor kernels, forked from stream
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    unsigned long long seed = 0;
    std::map<long long, long long> free_list;    // offset -> length (floats)
    std::vector<long long> off, len;
    std::vector<int> ns, active;
    std::vector<svpf_config_t> cfgs;
    std::vector<uint8_t> tiles;
    size_t smem1 = 0, smem2 = 0, smem2c = 0;
    int grid1 = 0, grid2 = 0, grid2c = 0;
    long long launches = 0;
    // device
    float* pool = nullptr;        // 4 arrays of pool_floats: h, h_prev, v, log_w
    int* d_n = nullptr;
    long long* d_off = nullptr;
    uint8_t* d_tile = nullptr;
    svpf_config_t* d_cfg = nullptr;
    SVPFParams* d_prm = nullptr;
    svpf_ctl_t* d_ctl = nullptr;
    int* d_queue = nullptr;
    int* d_req = nullptr;         // [cap] work list of a round (slots)
    float* d_y = nullptr;         // [cap]
    svpf_out_t* d_out = nullptr;  // [cap]
    int* h_req = nullptr;         // pinned staging
    float* h_y = nullptr;
    svpf_out_t* h_out = nullptr;
};

namespace {

template <class T>
bool salloc(T** p, size_t count, size_t* acc) {
    const size_t b = std::max<size_t>(count, 1) * sizeof(T);
    *acc += b;
    return cudaMalloc((void**)p, b) == cudaSuccess;
}

long long seg_len(int n, const svpf_config_t& c) { return ((c.use_two_factor ? 2LL : 1LL) * n + 15) / 16 * 16; }

double tick_cost(int n, const svpf_config_t& c) {
    if (c.use_two_factor) {
        const int na = c.use_annealing ? c.n_anneal_steps : 1;
        return 2.0 * n * n * std::max(na * c.n_stein_steps, 1);
    }
    return (double)n * n * std::max(c.stein_max_steps, 1);
}

void ctl_fresh(svpf_ctl_t* c) {
    std::memset(c, 0, sizeof(*c));
    c->ksd_prev = 1e10f;
    c->vol_prev = 0.05f;
    c->h_mean_prev = -3.5f;
    c->sigma_z_effective = 0.10f;
    c->mu_state = -3.5f;
    c->mu_var = 1.0f;
    for (int i = 0; i < SVPF_SMOOTH_MAX_LAG; ++i) c->smooth_h_var[i] = 1.0f;
}

BatchArgs round_args(svpf_stream* s) {
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = s->d_n;
    a.off = s->d_off;
    a.tile = s->d_tile;
    a.cfg = s->d_cfg;
    a.prm = s->d_prm;
    a.ctl = s->d_ctl;
    a.h = s->pool;
    a.hp = s->pool + s->pool_floats;
    a.v = s->pool + 2 * s->pool_floats;
    a.lw = s->pool + 3 * s->pool_floats;
    a.seed = s->seed;
    a.tape_stride = s->n_max;
    return a;
}

// Two-factor filters with at least this many particles take a cluster of
// kClusterMembers2f CTAs in the request loop: a round waits for its longest
// tick, and one CTA needs ~30 ms for an N = 2048 two-factor tick of 40 Stein
// steps.
constexpr int kClusterMinN = 1024;

bool big_2f(const svpf_stream* s, int slot) {
    return s->cfgs[slot].use_two_factor && s->ns[slot] >= kClusterMinN && s->grid2c > 0;
}

// One round: d_req[0, c1) single-factor slots, then c2 two-factor slots of
// which the first c2c run on clusters; each part largest cost first; y and
// outputs indexed alike.  The three kernels touch disjoint filters and have
// their own work counters, so they run concurrently: the clustered two-factor
// kernel (the longest ticks) and the one-CTA two-factor kernel on two side
// streams forked from the loop's stream, the single-factor kernel on the loop's
// stream, which then waits for both.  A kernel's CTAs take the SMs that another
// kernel's tail frees instead of waiting for the whole kernel to end.
int launch_round(svpf_stream* s, int c1, int c2, const int* d_req, const float* d_y, svpf_out_t* d_out,
                 int c2c = 0) {
    if (cudaMemsetAsync(s->d_queue, 0, 3 * sizeof(int), s->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    if (cudaEventRecord(s->fork, s->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    BatchArgs a = round_args(s);
    const int c2s = c2 - c2c;
    bool joined[2] = {false, false};
    if (c2c > 0) {
        a.F = c2c;
        a.order = d_req + c1;
        a.queue = s->d_queue + 2;
        a.req_y = d_y + c1;
        a.out = d_out + c1;
        if (cudaStreamWaitEvent(s->side[0], s->fork, 0) != cudaSuccess ||
            launch_batch_2f_cluster(a, s->smem2c, s->grid2c, s->side[0]) != cudaSuccess ||
            cudaEventRecord(s->join[0], s->side[0]) != cudaSuccess)
            return SVPF_ERR_CUDA;
        joined[0] = true;
        ++s->launches;
    }
    if (c2s > 0) {
        a.F = c2s;
        a.order = d_req + c1 + c2c;
        a.queue = s->d_queue + 1;
        a.req_y = d_y + c1 + c2c;
        a.out = d_out + c1 + c2c;
        if (cudaStreamWaitEvent(s->side[1], s->fork, 0) != cudaSuccess ||
            launch_batch_2f(a, s->smem2, s->grid2, s->side[1]) != cudaSuccess ||
            cudaEventRecord(s->join[1], s->side[1]) != cudaSuccess)
            return SVPF_ERR_CUDA;
        joined[1] = true;
        ++s->launches;
    }
    if (c1 > 0) {
        a.F = c1;
        a.order = d_req;
        a.queue = s->d_queue;
        a.req_y = d_y;
        a.out = d_out;
        if (launch_batch(a, s->smem1, s->grid1, s->stream) != cudaSuccess) return SVPF_ERR_CUDA;
        ++s->launches;
    }
    for (int k = 0; k < 2; ++k)
        if (joined[k] && cudaStreamWaitEvent(s->stream, s->join[k], 0) != cudaSuccess) return SVPF_ERR_CUDA;
    return SVPF_OK;
}

}  // namespace

extern "C" {

svpf_stream_t* svpf_stream_create(int max_instruments, size_t hbm_budget_bytes, int n_max, cudaStream_t stream) {
    SVPF_TRACE();
    if (max_instruments < 1 || n_max < 1 || n_max > SVPF_MAX_PARTICLES) return nullptr;
    svpf_stream* s = new svpf_stream();
    s->cap = max_instruments;
    s->n_max = n_max;
    s->budget = hbm_budget_bytes;
    const size_t C = (size_t)max_instruments;
    // per-instrument records and the request staging, then the particle pool
    const size_t fixed = C * (sizeof(int) + sizeof(long long) + 1 + sizeof(svpf_config_t) + sizeof(SVPFParams) +
                              sizeof(svpf_ctl_t) + sizeof(int) + sizeof(float) + sizeof(svpf_out_t)) + 64;
    if (hbm_budget_bytes <= fixed + 16 * 64) {
        delete s;
        return nullptr;
    }
    s->pool_floats = (hbm_budget_bytes - fixed) / (4 * sizeof(float)) / 16 * 16;
    if (stream) {
        s->stream = stream;
    } else {
        cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
        s->own_stream = true;
    }
    bool side_ok = true;
    for (int k = 0; k < 2; ++k) {
        side_ok = side_ok && cudaStreamCreateWithFlags(&s->side[k], cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&s->join[k], cudaEventDisableTiming) == cudaSuccess;
    }
    side_ok = side_ok && cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming) == cudaSuccess;
    if (!side_ok) {
        svpf_stream_destroy(s);
        return nullptr;
    }
    size_t acc = 0;
    bool ok = salloc(&s->pool, 4 * s->pool_floats, &acc) && salloc(&s->d_n, C, &acc) && salloc(&s->d_off, C, &acc) &&
              salloc(&s->d_tile, C, &acc) && salloc(&s->d_cfg, C, &acc) && salloc(&s->d_prm, C, &acc) &&
              salloc(&s->d_ctl, C, &acc) && salloc(&s->d_queue, 3, &acc) && salloc(&s->d_req, C, &acc) &&
              salloc(&s->d_y, C, &acc) && salloc(&s->d_out, C, &acc);
    s->fixed_bytes = acc - 4 * s->pool_floats * sizeof(float);
    ok = ok && cudaHostAlloc(&s->h_req, C * sizeof(int), cudaHostAllocDefault) == cudaSuccess &&
         cudaHostAlloc(&s->h_y, C * sizeof(float), cudaHostAllocDefault) == cudaSuccess &&
         cudaHostAlloc(&s->h_out, C * sizeof(svpf_out_t), cudaHostAllocDefault) == cudaSuccess;
    if (ok) {
        s->free_list[0] = (long long)s->pool_floats;
        s->off.assign(C, -1);
        s->len.assign(C, 0);
        s->ns.assign(C, 0);
        s->active.assign(C, 0);
        s->cfgs.resize(C);
        s->tiles.assign(C, 0);
        // shared memory sized for n_max; a model whose layout does not fit is
        // refused at admission
        s->smem1 = tick_smem_bytes(n_max, 1, false);
        s->smem2 = tick_smem_bytes_2f(n_max, 1);
        if (s->smem1 <= max_dyn_smem()) s->grid1 = batch_grid(s->smem1);
        if (s->smem2 <= max_dyn_smem()) s->grid2 = batch_grid_2f(s->smem2);
        s->smem2c = tick_smem_bytes_2f(n_max, kClusterMembers2f);
        if (n_max >= kClusterMinN && s->smem2c <= max_dyn_smem()) s->grid2c = batch_cluster_grid_2f(s->smem2c);
        ok = s->grid1 > 0 || s->grid2 > 0;
    }
    if (!ok) {
        svpf_stream_destroy(s);
        return nullptr;
    }
    return s;
}

void svpf_stream_destroy(svpf_stream_t* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    void* ptrs[] = {s->pool, s->d_n, s->d_off, s->d_tile, s->d_cfg, s->d_prm, s->d_ctl, s->d_queue, s->d_req,
                    s->d_y, s->d_out};
    for (void* p : ptrs) cudaFree(p);
    if (s->h_req) cudaFreeHost(s->h_req);
    if (s->h_y) cudaFreeHost(s->h_y);
    if (s->h_out) cudaFreeHost(s->h_out);
    for (int k = 0; k < 2; ++k) {
        if (s->side[k]) {
            cudaStreamSynchronize(s->side[k]);
            cudaStreamDestroy(s->side[k]);
        }
        if (s->join[k]) cudaEventDestroy(s->join[k]);
    }
    if (s->fork) cudaEventDestroy(s->fork);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
}

void svpf_stream_set_seed(svpf_stream_t* s, unsigned long long seed) {
    if (s) s->seed = seed;
}

int svpf_stream_admit(svpf_stream_t* s, int n, const svpf_config_t* cfg, const SVPFParams* p,
                      unsigned long long seed) {
    SVPF_TRACE();
    if (!s || !cfg || !p || n < 1 || n > s->n_max) return -SVPF_ERR_INVALID_ARG;
    if (cfg->use_heun) return -SVPF_ERR_UNSUPPORTED;   // the loop's shared-memory layout has no Heun buffers
    if (!cfg->use_two_factor && s->grid1 < 1) return -SVPF_ERR_UNSUPPORTED;
    if (cfg->use_two_factor && s->grid2 < 1 && !(n >= kClusterMinN && s->grid2c > 0)) return -SVPF_ERR_UNSUPPORTED;
    if (cfg->use_two_factor && cfg->n_stein_steps < 1) return -SVPF_ERR_INVALID_ARG;
    if (!config_loops_ok(*cfg)) return -SVPF_ERR_INVALID_ARG;
    int slot = -1;
    for (int i = 0; i < s->cap; ++i)
        if (!s->active[i]) { slot = i; break; }
    if (slot < 0) return -SVPF_ERR_BUDGET;
    const long long L = seg_len(n, *cfg);
    long long at = -1;
    for (auto it = s->free_list.begin(); it != s->free_list.end(); ++it) {
        if (it->second >= L) {
            at = it->first;
            const long long rest = it->second - L;
            s->free_list.erase(it);
            if (rest > 0) s->free_list[at + L] = rest;
            break;
        }
    }
    if (at < 0) return -SVPF_ERR_BUDGET;
    s->active[slot] = 1;
    s->off[slot] = at;
    s->len[slot] = L;
    s->ns[slot] = n;
    s->cfgs[slot] = *cfg;
    s->used_floats += (size_t)L;
    {
        const int t = tuned_batch_tile(n);
        s->tiles[slot] = (uint8_t)(t >= kBatchTileLo && t <= kBatchTileHi ? t : default_batch_tile(n));
    }
    // control record as svpf_initialize leaves it (svpf_optimized_graph.cu:349-451)
    svpf_config_t c = *cfg;
    c.nu_state = std::max(c.nu_state, 2.5f);
    const float base_var = p->sigma_z * p->sigma_z / (1.0f - p->rho * p->rho + 1e-6f);
    const float var = c.use_student_t_state ? c.nu_state / (c.nu_state - 2.0f) * base_var : base_var;
    svpf_ctl_t ctl;
    ctl_fresh(&ctl);
    ctl.guide_mean = p->mu;
    ctl.guide_var = var;
    if (c.use_adaptive_mu) { ctl.mu_state = p->mu; ctl.mu_var = 1.0f; }
    if (c.use_adaptive_sigma) ctl.sigma_z_effective = p->sigma_z;
    ctl.stein_steps_used = c.n_stein_steps;
    if (c.use_two_factor) {
        ctl.guide_var_fast = c.sigma_fast * c.sigma_fast / (1.0f - c.rho_fast * c.rho_fast + 1e-6f);
        ctl.guide_var_slow = c.sigma_slow * c.sigma_slow / (1.0f - c.rho_slow * c.rho_slow + 1e-6f);
    }
    const long long off = at;
    cudaError_t e = cudaMemcpyAsync(s->d_n + slot, &s->ns[slot], sizeof(int), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_off + slot, &s->off[slot], sizeof(long long), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_tile + slot, &s->tiles[slot], 1, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_cfg + slot, &c, sizeof(c), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_prm + slot, p, sizeof(SVPFParams), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_ctl + slot, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->pool + 3 * s->pool_floats + off, 0, L * sizeof(float), s->stream);
    InitArgs a;
    std::memset(&a, 0, sizeof(a));
    a.h = s->pool + off;
    a.hp = s->pool + s->pool_floats + off;
    a.v = s->pool + 2 * s->pool_floats + off;
    a.n0 = n;
    a.F = 1;
    a.mu0 = p->mu;
    a.sd0 = sqrtf(var);
    a.seed = seed;
    a.key_base = slot;   // initial draws keyed by (seed, slot), as a batch keys filter f by (seed, f)
    a.tape_stride = n;
    if (c.use_two_factor) {
        a.tf0 = 1;
        a.sdf0 = c.sigma_fast / sqrtf(1.0f - c.rho_fast * c.rho_fast + 1e-8f);
        a.sds0 = c.sigma_slow / sqrtf(1.0f - c.rho_slow * c.rho_slow + 1e-8f);
    }
    if (e == cudaSuccess) e = launch_init(a, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);   // the host records above are stack values
    if (e != cudaSuccess) {
        svpf_stream_evict(s, slot);
        return -SVPF_ERR_CUDA;
    }
    return slot;
}

int svpf_stream_evict(svpf_stream_t* s, int slot) {
    SVPF_TRACE();
    if (!s || slot < 0 || slot >= s->cap || !s->active[slot]) return SVPF_ERR_INVALID_ARG;
    cudaStreamSynchronize(s->stream);
    long long at = s->off[slot], L = s->len[slot];
    // return the segment, merging with free neighbours
    auto next = s->free_list.lower_bound(at);
    if (next != s->free_list.end() && next->first == at + L) {
        L += next->second;
        next = s->free_list.erase(next);
    }
    if (next != s->free_list.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == at) {
            at = prev->first;
            L += prev->second;
            s->free_list.erase(prev);
        }
    }
    s->free_list[at] = L;
    s->used_floats -= (size_t)s->len[slot];
    s->active[slot] = 0;
    s->off[slot] = -1;
    s->len[slot] = 0;
    return SVPF_OK;
}

size_t svpf_stream_bytes_in_use(const svpf_stream_t* s) {
    return s ? s->fixed_bytes + 4 * s->used_floats * sizeof(float) : 0;
}

size_t svpf_stream_bytes_budget(const svpf_stream_t* s) { return s ? s->budget : 0; }

int svpf_stream_process(svpf_stream_t* s, int count, const int* slots, const float* y, svpf_out_t* out) {
    SVPF_TRACE();
    if (!s || count < 0 || (count > 0 && (!slots || !y))) return SVPF_ERR_INVALID_ARG;
    for (int r = 0; r < count; ++r)
        if (slots[r] < 0 || slots[r] >= s->cap || !s->active[slots[r]]) return SVPF_ERR_INVALID_ARG;
    // rounds: the k-th request of an instrument goes to round k
    std::vector<int> seen(s->cap, 0), round(count);
    int rounds = 0;
    for (int r = 0; r < count; ++r) {
        round[r] = seen[slots[r]]++;
        rounds = std::max(rounds, round[r] + 1);
    }
    std::vector<int> idx;
    std::vector<std::vector<int>> where(rounds);
    for (int r = 0; r < count; ++r) where[round[r]].push_back(r);
    for (int k = 0; k < rounds; ++k) {
        idx = where[k];
        // single-factor, then two-factor on clusters, then two-factor on one
        // CTA; each part largest cost first
        auto group = [&](int r) { return !s->cfgs[slots[r]].use_two_factor ? 0 : (big_2f(s, slots[r]) ? 1 : 2); };
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
            if (group(a) != group(b)) return group(a) < group(b);
            return tick_cost(s->ns[slots[a]], s->cfgs[slots[a]]) > tick_cost(s->ns[slots[b]], s->cfgs[slots[b]]);
        });
        int c1 = 0, c2c = 0;
        for (size_t q = 0; q < idx.size(); ++q) {
            s->h_req[q] = slots[idx[q]];
            s->h_y[q] = y[idx[q]];
            const int gq = group(idx[q]);
            if (gq == 0) ++c1;
            if (gq == 1) ++c2c;
        }
        const int m = (int)idx.size();
        if (cudaMemcpyAsync(s->d_req, s->h_req, m * sizeof(int), cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
            cudaMemcpyAsync(s->d_y, s->h_y, m * sizeof(float), cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
            return SVPF_ERR_CUDA;
        const int rc = launch_round(s, c1, m - c1, s->d_req, s->d_y, s->d_out, c2c);
        if (rc != SVPF_OK) return rc;
        if (cudaMemcpyAsync(s->h_out, s->d_out, m * sizeof(svpf_out_t), cudaMemcpyDeviceToHost, s->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess)
            return SVPF_ERR_CUDA;
        if (out)
            for (int q = 0; q < m; ++q) out[idx[q]] = s->h_out[q];
    }
    return SVPF_OK;
}

int svpf_stream_process_device(svpf_stream_t* s, int count1, int count2, const int* d_slots, const float* d_y,
                               svpf_out_t* d_out) {
    SVPF_TRACE();
    if (!s || count1 < 0 || count2 < 0 || count1 + count2 > s->cap || !d_slots || !d_y || !d_out)
        return SVPF_ERR_INVALID_ARG;
    if (count1 + count2 == 0) return SVPF_OK;
    return launch_round(s, count1, count2, d_slots, d_y, d_out);
}

int svpf_stream_get_ctl(const svpf_stream_t* s, int slot, svpf_ctl_t* ctl) {
    if (!s || !ctl || slot < 0 || slot >= s->cap || !s->active[slot]) return SVPF_ERR_INVALID_ARG;
    cudaStreamSynchronize(s->stream);
    return cudaMemcpy(ctl, s->d_ctl + slot, sizeof(svpf_ctl_t), cudaMemcpyDeviceToHost) == cudaSuccess ? SVPF_OK
                                                                                                     : SVPF_ERR_CUDA;
}

int svpf_stream_get_particles(const svpf_stream_t* s, int slot, float* h_out) {
    if (!s || !h_out || slot < 0 || slot >= s->cap || !s->active[slot]) return SVPF_ERR_INVALID_ARG;
    cudaStreamSynchronize(s->stream);
    const size_t len = (size_t)(s->cfgs[slot].use_two_factor ? 2 : 1) * s->ns[slot];
    return cudaMemcpy(h_out, s->pool + s->off[slot], len * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess
               ? SVPF_OK : SVPF_ERR_CUDA;
}

long long svpf_stream_kernel_launches(const svpf_stream_t* s) { return s ? s->launches : 0; }

}  // extern "C"
