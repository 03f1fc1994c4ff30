// svpf_batch.cu -- batch API: many independent filters, one persistent launch
// per tick.
//
// HBM layout: the particle arrays of all filters are packed back to back
// (filter f at offset off[f], n[f] floats -- 2 n[f] for a two-factor filter,
// fast then slow -- offsets rounded to 16 floats), one packed array each for
// h, h_prev, v and log_w.  Per-filter configuration, parameters and control
// records are arrays of structs.  Single-factor and two-factor filters run in
// two persistent kernels, one after the other on the batch's stream; each
// takes its filters from a work counter in decreasing order of cost (n^2 times
// the Stein budget bound), so the largest ticks start first.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <utility>
#include <vector>

#include "svpf.h"
#include "svpf_internal.h"
#include "svpf_trace.h"

using namespace svpf;

struct svpf_batch {
    int F = 0;
    int F1 = 0, F2 = 0;          // single-factor / two-factor filters
    int n_max = 0;
    int n_max1 = 0, n_max2 = 0;
    std::vector<uint8_t> tf;     // two-factor flag per filter
    long long total = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<int> ns;
    std::vector<long long> offs;
    std::vector<svpf_config_t> cfgs;
    std::vector<SVPFParams> prms;
    std::vector<uint8_t> tiles;
    // device
    int* d_n = nullptr;
    long long* d_off = nullptr;
    uint8_t* d_tile = nullptr;
    int* d_order = nullptr;
    int* d_queue = nullptr;
    svpf_config_t* d_cfg = nullptr;
    SVPFParams* d_prm = nullptr;
    svpf_ctl_t* d_ctl = nullptr;
    float* d_h = nullptr;
    float* d_hp = nullptr;
    float* d_v = nullptr;
    float* d_lw = nullptr;
    float* d_y = nullptr;        // [2F] staging: y_t then y_prev
    svpf_out_t* d_out = nullptr;
    float* h_stage = nullptr;    // pinned [2F]
    svpf_out_t* h_out = nullptr; // pinned [F]
    float* tape_n = nullptr;
    float* tape_u = nullptr;
    int slots_n = 0, slots_u = 0;
    unsigned long long seed = 0;
    size_t smem = 0, smem2 = 0;
    int grid = 0, grid2 = 0;
    int launches = 0;
    int heun = 0;
    int prod = 0;                // every single-factor filter has the production configuration
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const float* g_yt = nullptr;
    const float* g_yp = nullptr;
    svpf_out_t* g_out = nullptr;
};

namespace {

template <class T>
bool dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T)) == cudaSuccess;
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

BatchArgs make_args(svpf_batch* b, const float* d_yt, const float* d_yp, svpf_out_t* d_out) {
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.F = b->F1;
    a.order = b->d_order;
    a.queue = b->d_queue;
    a.n = b->d_n;
    a.off = b->d_off;
    a.tile = b->d_tile;
    a.cfg = b->d_cfg;
    a.prm = b->d_prm;
    a.ctl = b->d_ctl;
    a.h = b->d_h;
    a.hp = b->d_hp;
    a.v = b->d_v;
    a.lw = b->d_lw;
    a.y_t = d_yt;
    a.y_prev = d_yp;
    a.out = d_out;
    a.seed = b->seed;
    a.tape_n = b->tape_n;
    a.tape_u = b->tape_u;
    a.slots_n = b->slots_n;
    a.slots_u = b->slots_u;
    a.tape_stride = b->n_max;
    a.heun = b->heun;
    a.prod = b->prod;
    return a;
}

int kernels_per_tick(const svpf_batch* b) { return (b->F1 > 0 ? 1 : 0) + (b->F2 > 0 ? 1 : 0); }

int enqueue_tick(svpf_batch* b, const float* d_yt, const float* d_yp, svpf_out_t* d_out) {
    if (cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(int), b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    BatchArgs a = make_args(b, d_yt, d_yp, d_out);
    if (b->F1 > 0) {
        if (launch_batch(a, b->smem, b->grid, b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
        ++b->launches;
    }
    if (b->F2 > 0) {
        a.F = b->F2;
        a.order = b->d_order + b->F1;
        a.queue = b->d_queue + 1;
        if (launch_batch_2f(a, b->smem2, b->grid2, b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
        ++b->launches;
    }
    return SVPF_OK;
}

void drop_graph(svpf_batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

int upload_tiles(svpf_batch* b) {
    for (int f = 0; f < b->F; ++f) {
        const int t = tuned_batch_tile(b->ns[f]);
        b->tiles[f] = (uint8_t)(t >= kBatchTileLo && t <= kBatchTileHi ? t : default_batch_tile(b->ns[f]));
    }
    return cudaMemcpy(b->d_tile, b->tiles.data(), b->F, cudaMemcpyHostToDevice) == cudaSuccess ? SVPF_OK
                                                                                              : SVPF_ERR_CUDA;
}

}  // namespace

extern "C" {

svpf_batch_t* svpf_batch_create(int F, const int* ns, const svpf_config_t* cfgs, const SVPFParams* prms,
                                cudaStream_t stream) {
    SVPF_TRACE();
    if (F < 1 || !ns || !cfgs || !prms) return nullptr;
    int n_max = 0, n_max1 = 0, n_max2 = 0, F1 = 0, heun = 0, prod = 1;
    for (int f = 0; f < F; ++f) {
        if (ns[f] < 1 || ns[f] > SVPF_MAX_PARTICLES || !config_loops_ok(cfgs[f])) return nullptr;
        n_max = std::max(n_max, ns[f]);
        if (cfgs[f].use_two_factor) {
            if (cfgs[f].n_stein_steps < 1) return nullptr;
            n_max2 = std::max(n_max2, ns[f]);
        } else {
            n_max1 = std::max(n_max1, ns[f]);
            heun |= cfgs[f].use_heun != 0;
            prod &= is_production_tick(cfgs[f]) ? 1 : 0;
            ++F1;
        }
    }
    if (F1 > 0 && tick_smem_bytes(n_max1, 1, heun != 0) > max_dyn_smem()) return nullptr;
    if (F1 < F && tick_smem_bytes_2f(n_max2, 1) > max_dyn_smem()) return nullptr;
    svpf_batch* b = new svpf_batch();
    b->heun = heun;
    b->prod = prod;
    b->F = F;
    b->F1 = F1;
    b->F2 = F - F1;
    b->n_max = n_max;
    b->n_max1 = n_max1;
    b->n_max2 = n_max2;
    b->tf.resize(F);
    for (int f = 0; f < F; ++f) b->tf[f] = cfgs[f].use_two_factor ? 1 : 0;
    b->ns.assign(ns, ns + F);
    b->cfgs.assign(cfgs, cfgs + F);
    b->prms.assign(prms, prms + F);
    b->tiles.assign(F, 0);
    b->offs.resize(F);
    long long off = 0;
    for (int f = 0; f < F; ++f) {
        b->offs[f] = off;
        off += ((b->tf[f] ? 2 : 1) * ns[f] + 15) / 16 * 16;
    }
    b->total = off;
    if (stream) {
        b->stream = stream;
    } else {
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        b->own_stream = true;
    }
    // work order: single-factor filters then two-factor filters, each
    // largest expected cost first
    auto cost = [&](int f) {
        const svpf_config_t& c = cfgs[f];
        if (c.use_two_factor) {
            const int na = c.use_annealing ? c.n_anneal_steps : 1;
            return 2.0 * ns[f] * ns[f] * std::max(na * c.n_stein_steps, 1);
        }
        return (double)ns[f] * ns[f] * std::max(c.stein_max_steps, 1);
    };
    std::vector<int> order(F);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        if (b->tf[a] != b->tf[c]) return b->tf[a] < b->tf[c];
        return cost(a) > cost(c);
    });
    std::vector<svpf_ctl_t> ctl(F);
    for (auto& c : ctl) ctl_fresh(&c);
    bool ok = dalloc(&b->d_n, F) && dalloc(&b->d_off, F) && dalloc(&b->d_tile, F) && dalloc(&b->d_order, F) &&
              dalloc(&b->d_queue, 2) && dalloc(&b->d_cfg, F) && dalloc(&b->d_prm, F) && dalloc(&b->d_ctl, F) &&
              dalloc(&b->d_h, b->total) && dalloc(&b->d_hp, b->total) && dalloc(&b->d_v, b->total) &&
              dalloc(&b->d_lw, b->total) && dalloc(&b->d_y, 2 * (size_t)F) && dalloc(&b->d_out, F);
    ok = ok && cudaHostAlloc(&b->h_stage, 2 * (size_t)F * sizeof(float), cudaHostAllocDefault) == cudaSuccess &&
         cudaHostAlloc(&b->h_out, (size_t)F * sizeof(svpf_out_t), cudaHostAllocDefault) == cudaSuccess;
    ok = ok && cudaMemcpy(b->d_n, ns, F * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(b->d_off, b->offs.data(), F * sizeof(long long), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(b->d_order, order.data(), F * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(b->d_cfg, cfgs, F * sizeof(svpf_config_t), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(b->d_prm, prms, F * sizeof(SVPFParams), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(b->d_ctl, ctl.data(), F * sizeof(svpf_ctl_t), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(b->d_lw, 0, b->total * sizeof(float)) == cudaSuccess;
    ok = ok && upload_tiles(b) == SVPF_OK;
    if (ok && b->F1 > 0) {
        b->smem = tick_smem_bytes(n_max1, 1, heun != 0);
        b->grid = batch_grid(b->smem);
        ok = b->grid > 0;
    }
    if (ok && b->F2 > 0) {
        b->smem2 = tick_smem_bytes_2f(n_max2, 1);
        b->grid2 = batch_grid_2f(b->smem2);
        ok = b->grid2 > 0;
    }
    if (!ok) {
        svpf_batch_destroy(b);
        return nullptr;
    }
    return b;
}

void svpf_batch_destroy(svpf_batch_t* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    cudaFree(b->d_n);
    cudaFree(b->d_off);
    cudaFree(b->d_tile);
    cudaFree(b->d_order);
    cudaFree(b->d_queue);
    cudaFree(b->d_cfg);
    cudaFree(b->d_prm);
    cudaFree(b->d_ctl);
    cudaFree(b->d_h);
    cudaFree(b->d_hp);
    cudaFree(b->d_v);
    cudaFree(b->d_lw);
    cudaFree(b->d_y);
    cudaFree(b->d_out);
    if (b->tape_n) cudaFree(b->tape_n);
    if (b->tape_u) cudaFree(b->tape_u);
    if (b->h_stage) cudaFreeHost(b->h_stage);
    if (b->h_out) cudaFreeHost(b->h_out);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
}

// svpf_initialize for every filter (svpf_optimized_graph.cu:349-451)
int svpf_batch_initialize(svpf_batch_t* b, unsigned long long seed) {
    SVPF_TRACE();
    if (!b) return SVPF_ERR_INVALID_ARG;
    b->seed = seed;
    if (b->F2 > 0 && b->tape_n && b->slots_n < 3) return SVPF_ERR_TAPE_SHORT;
    std::vector<float> mu(b->F), sd(b->F), sdf(b->F, 0.0f), sds(b->F, 0.0f);
    std::vector<svpf_ctl_t> ctl(b->F);
    if (cudaMemcpy(ctl.data(), b->d_ctl, b->F * sizeof(svpf_ctl_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SVPF_ERR_CUDA;
    for (int f = 0; f < b->F; ++f) {
        svpf_config_t& c = b->cfgs[f];
        const SVPFParams& p = b->prms[f];
        c.nu_state = std::max(c.nu_state, 2.5f);
        const float base_var = p.sigma_z * p.sigma_z / (1.0f - p.rho * p.rho + 1e-6f);
        const float var = c.use_student_t_state ? c.nu_state / (c.nu_state - 2.0f) * base_var : base_var;
        mu[f] = p.mu;
        sd[f] = std::sqrt(var);
        svpf_ctl_t& s = ctl[f];
        s.timestep = 0;
        s.y_prev = 0.0f;
        s.guide_initialized = 0;
        s.guide_mean = p.mu;
        s.guide_var = var;
        if (c.use_adaptive_mu) {
            s.mu_state = p.mu;
            s.mu_var = 1.0f;
        }
        if (c.use_adaptive_sigma) s.sigma_z_effective = p.sigma_z;
        s.ksd_prev = 1e10f;
        s.stein_steps_used = c.n_stein_steps;
        s.loglik_sum = 0.0;
        s.status = SVPF_OK;
        if (c.use_two_factor) {
            // svpf_optimized_graph.cu:414-447; the factor means of the previous
            // tick (the guide's reference point) are kept, as the reference does
            sdf[f] = c.sigma_fast / std::sqrt(1.0f - c.rho_fast * c.rho_fast + 1e-8f);
            sds[f] = c.sigma_slow / std::sqrt(1.0f - c.rho_slow * c.rho_slow + 1e-8f);
            s.guide_2f_initialized = 0;
            s.guide_mean_fast = 0.0;
            s.guide_mean_slow = 0.0;
            s.guide_var_fast = c.sigma_fast * c.sigma_fast / (1.0f - c.rho_fast * c.rho_fast + 1e-6f);
            s.guide_var_slow = c.sigma_slow * c.sigma_slow / (1.0f - c.rho_slow * c.rho_slow + 1e-6f);
        }
    }
    float *d_mu = nullptr, *d_sd = nullptr, *d_sdf = nullptr, *d_sds = nullptr;
    uint8_t* d_tf = nullptr;
    if (!dalloc(&d_mu, b->F) || !dalloc(&d_sd, b->F) || !dalloc(&d_sdf, b->F) || !dalloc(&d_sds, b->F) ||
        !dalloc(&d_tf, b->F)) {
        cudaFree(d_mu);
        cudaFree(d_sd);
        cudaFree(d_sdf);
        cudaFree(d_sds);
        cudaFree(d_tf);
        return SVPF_ERR_CUDA;
    }
    const bool copied =
        cudaMemcpy(d_mu, mu.data(), b->F * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(d_sd, sd.data(), b->F * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(d_sdf, sdf.data(), b->F * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(d_sds, sds.data(), b->F * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(d_tf, b->tf.data(), b->F, cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(b->d_cfg, b->cfgs.data(), b->F * sizeof(svpf_config_t), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(b->d_ctl, ctl.data(), b->F * sizeof(svpf_ctl_t), cudaMemcpyHostToDevice) == cudaSuccess;
    InitArgs a;
    std::memset(&a, 0, sizeof(a));
    a.h = b->d_h;
    a.hp = b->d_hp;
    a.v = b->d_v;
    a.off = b->d_off;
    a.n = b->d_n;
    a.F = b->F;
    a.mu = d_mu;
    a.sd = d_sd;
    a.seed = seed;
    a.tape0 = b->tape_n;   // test tape: slot 0 (and 1, 2 for two factors) hold the initial normals
    a.tape_stride = b->n_max;
    a.tf = d_tf;
    a.sdf = d_sdf;
    a.sds = d_sds;
    cudaError_t e = copied ? launch_init(a, b->stream) : cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(d_mu);
    cudaFree(d_sd);
    cudaFree(d_sdf);
    cudaFree(d_sds);
    cudaFree(d_tf);
    return e == cudaSuccess ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_batch_step(svpf_batch_t* b, const float* y_t, const float* y_prev, float* loglik, float* vol,
                    float* h_mean) {
    SVPF_TRACE();
    if (!b || !y_t || !y_prev) return SVPF_ERR_INVALID_ARG;
    const size_t F = (size_t)b->F;
    std::memcpy(b->h_stage, y_t, F * sizeof(float));
    std::memcpy(b->h_stage + F, y_prev, F * sizeof(float));
    if (cudaMemcpyAsync(b->d_y, b->h_stage, 2 * F * sizeof(float), cudaMemcpyHostToDevice, b->stream) !=
        cudaSuccess)
        return SVPF_ERR_CUDA;
    int rc = enqueue_tick(b, b->d_y, b->d_y + F, b->d_out);
    if (rc != SVPF_OK) return rc;
    if (cudaMemcpyAsync(b->h_out, b->d_out, F * sizeof(svpf_out_t), cudaMemcpyDeviceToHost, b->stream) !=
        cudaSuccess)
        return SVPF_ERR_CUDA;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    for (size_t f = 0; f < F; ++f) {
        if (loglik) loglik[f] = b->h_out[f].loglik;
        if (vol) vol[f] = b->h_out[f].vol;
        if (h_mean) h_mean[f] = b->h_out[f].h_mean;
    }
    return SVPF_OK;
}

int svpf_batch_step_device(svpf_batch_t* b, const float* d_yt, const float* d_yp, svpf_out_t* d_out) {
    SVPF_TRACE();
    if (!b || !d_yt || !d_yp) return SVPF_ERR_INVALID_ARG;
    return enqueue_tick(b, d_yt, d_yp, d_out);
}

int svpf_batch_graph_launch(svpf_batch_t* b, const float* d_yt, const float* d_yp, svpf_out_t* d_out) {
    SVPF_TRACE();
    if (!b || !d_yt || !d_yp) return SVPF_ERR_INVALID_ARG;
    if (b->gexec && (b->g_yt != d_yt || b->g_yp != d_yp || b->g_out != d_out)) drop_graph(b);
    if (!b->gexec) {
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return SVPF_ERR_CUDA;
        const int launches = b->launches;
        const int rc = enqueue_tick(b, d_yt, d_yp, d_out);
        b->launches = launches;   // counted per replay below
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc != SVPF_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return SVPF_ERR_CUDA;
        }
        if (cudaGraphInstantiate(&b->gexec, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            return SVPF_ERR_CUDA;
        }
        b->graph = g;
        b->g_yt = d_yt;
        b->g_yp = d_yp;
        b->g_out = d_out;
    }
    if (cudaGraphLaunch(b->gexec, b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    b->launches += kernels_per_tick(b);
    return SVPF_OK;
}

int svpf_batch_sync(svpf_batch_t* b) {
    if (!b) return SVPF_ERR_INVALID_ARG;
    return cudaStreamSynchronize(b->stream) == cudaSuccess ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_batch_n_filters(const svpf_batch_t* b) { return b ? b->F : 0; }

int svpf_batch_get_config(const svpf_batch_t* b, int f, svpf_config_t* cfg) {
    if (!b || !cfg || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    *cfg = b->cfgs[f];
    return SVPF_OK;
}

int svpf_batch_last_outputs(const svpf_batch_t* b, svpf_out_t* out) {
    if (!b || !out) return SVPF_ERR_INVALID_ARG;
    std::memcpy(out, b->h_out, (size_t)b->F * sizeof(svpf_out_t));   // filled by svpf_batch_step
    return SVPF_OK;
}
int svpf_batch_kernel_launches(const svpf_batch_t* b) { return b ? b->launches : 0; }

int svpf_batch_get_ctl(const svpf_batch_t* b, svpf_ctl_t* ctl) {
    if (!b || !ctl) return SVPF_ERR_INVALID_ARG;
    cudaStreamSynchronize(b->stream);
    return cudaMemcpy(ctl, b->d_ctl, b->F * sizeof(svpf_ctl_t), cudaMemcpyDeviceToHost) == cudaSuccess
               ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_batch_get_particles(const svpf_batch_t* b, int f, float* h_out) {
    if (!b || !h_out || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    cudaStreamSynchronize(b->stream);
    const size_t len = (size_t)(b->tf[f] ? 2 : 1) * b->ns[f];
    return cudaMemcpy(h_out, b->d_h + b->offs[f], len * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess
               ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_batch_get_params(const svpf_batch_t* b, int f, SVPFParams* p) {
    if (!b || !p || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    *p = b->prms[f];
    return SVPF_OK;
}

int svpf_batch_set_params(svpf_batch_t* b, int f, const SVPFParams* p) {
    if (!b || !p || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    b->prms[f] = *p;
    // stream ordered: ticks already enqueued keep the old parameters
    return cudaMemcpyAsync(b->d_prm + f, &b->prms[f], sizeof(SVPFParams), cudaMemcpyHostToDevice, b->stream) ==
                   cudaSuccess && cudaStreamSynchronize(b->stream) == cudaSuccess
               ? SVPF_OK : SVPF_ERR_CUDA;
}

int svpf_batch_get_state(const svpf_batch_t* b, int f, svpf_ctl_t* ctl, float* h, float* hp, float* v, float* lw) {
    if (!b || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    const size_t len = (size_t)(b->tf[f] ? 2 : 1) * b->ns[f], off = (size_t)b->offs[f];
    const std::pair<float*, const float*> arrs[] = {{h, b->d_h}, {hp, b->d_hp}, {v, b->d_v}};
    for (const auto& a : arrs)
        if (a.first && cudaMemcpy(a.first, a.second + off, len * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            return SVPF_ERR_CUDA;
    if (lw && cudaMemcpy(lw, b->d_lw + off, b->ns[f] * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SVPF_ERR_CUDA;
    if (ctl && cudaMemcpy(ctl, b->d_ctl + f, sizeof(svpf_ctl_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SVPF_ERR_CUDA;
    return SVPF_OK;
}

int svpf_batch_set_state(svpf_batch_t* b, int f, const svpf_ctl_t* ctl, const float* h, const float* hp,
                         const float* v, const float* lw) {
    if (!b || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    const size_t len = (size_t)(b->tf[f] ? 2 : 1) * b->ns[f], off = (size_t)b->offs[f];
    const std::pair<const float*, float*> arrs[] = {{h, b->d_h}, {hp, b->d_hp}, {v, b->d_v}};
    for (const auto& a : arrs)
        if (a.first && cudaMemcpy(a.second + off, a.first, len * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
            return SVPF_ERR_CUDA;
    if (lw && cudaMemcpy(b->d_lw + off, lw, b->ns[f] * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return SVPF_ERR_CUDA;
    if (ctl && cudaMemcpy(b->d_ctl + f, ctl, sizeof(svpf_ctl_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return SVPF_ERR_CUDA;
    return SVPF_OK;
}

int svpf_batch_set_noise_tape(svpf_batch_t* b, const float* normals, int ns, const float* uniforms, int nu_) {
    if (!b) return SVPF_ERR_INVALID_ARG;
    if (b->tape_n) cudaFree(b->tape_n);
    if (b->tape_u) cudaFree(b->tape_u);
    b->tape_n = b->tape_u = nullptr;
    b->slots_n = b->slots_u = 0;
    drop_graph(b);
    if (!normals) return SVPF_OK;
    if (ns < 1 || nu_ < 1 || !uniforms) return SVPF_ERR_INVALID_ARG;
    const size_t w = (size_t)b->n_max;
    if (!dalloc(&b->tape_n, ns * w) || !dalloc(&b->tape_u, nu_ * w)) return SVPF_ERR_CUDA;
    if (cudaMemcpy(b->tape_n, normals, ns * w * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->tape_u, uniforms, nu_ * w * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return SVPF_ERR_CUDA;
    b->slots_n = ns;
    b->slots_u = nu_;
    return SVPF_OK;
}

int svpf_batch_tile_of(const svpf_batch_t* b, int n, int* R, int* S) {
    if (!b) return SVPF_ERR_INVALID_ARG;
    for (int f = 0; f < b->F; ++f) {
        if (b->ns[f] == n) {
            if (R) *R = kTiles[b->tiles[f]].R;
            if (S) *S = kTiles[b->tiles[f]].S;
            return SVPF_OK;
        }
    }
    if (R) *R = -1;
    if (S) *S = -1;
    return SVPF_ERR_INVALID_ARG;
}

// Autotuner: for each particle count, time every batch tile shape on a
// synthetic batch that fills the GPU (one filter per resident CTA) and keep
// the fastest.  Production configuration, fixed budget (stein_min = max).
// Any failed call (allocation, copy, launch, a tile's tick) ends the tuning
// with SVPF_ERR_CUDA and records no choice for that size.
namespace {

int tune_one(int n, int ticks, int* best_tile) {
    const size_t smem = tick_smem_bytes(n, 1, false);
    if (smem > max_dyn_smem()) return SVPF_ERR_INVALID_ARG;
    const int F = batch_grid(smem);
    if (F < 1) return SVPF_ERR_CUDA;
    svpf_config_t c;
    svpf_config_init(&c, 8, 30.0f);
    c.use_newton = 1;
    c.use_full_newton = 1;
    c.stein_min_steps = 8;
    c.stein_max_steps = 8;
    std::vector<int> nv(F, n);
    std::vector<svpf_config_t> cv(F, c);
    std::vector<SVPFParams> pv(F, SVPFParams{0.97f, 0.15f, -1.0f, 0.0f});
    svpf_batch_t* b = svpf_batch_create(F, nv.data(), cv.data(), pv.data(), nullptr);
    if (!b) return SVPF_ERR_CUDA;
    float* d_y = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = svpf_batch_initialize(b, 1234);
    if (rc == SVPF_OK && !dalloc(&d_y, 2 * (size_t)F)) rc = SVPF_ERR_CUDA;
    if (rc == SVPF_OK) {
        std::vector<float> ys(2 * (size_t)F);
        std::fill(ys.begin(), ys.begin() + F, 0.3f);
        std::fill(ys.begin() + F, ys.end(), 0.2f);
        if (cudaMemcpy(d_y, ys.data(), ys.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
            rc = SVPF_ERR_CUDA;
    }
    float best = 1e30f;
    int best_t = -1;
    for (int t = kBatchTileLo; rc == SVPF_OK && t <= kBatchTileHi; ++t) {
        std::fill(b->tiles.begin(), b->tiles.end(), (uint8_t)t);
        if (cudaMemcpy(b->d_tile, b->tiles.data(), F, cudaMemcpyHostToDevice) != cudaSuccess) {
            rc = SVPF_ERR_CUDA;
            break;
        }
        rc = enqueue_tick(b, d_y, d_y + F, nullptr);   // warm
        if (rc == SVPF_OK && cudaEventRecord(e0, b->stream) != cudaSuccess) rc = SVPF_ERR_CUDA;
        for (int i = 0; rc == SVPF_OK && i < ticks; ++i) rc = enqueue_tick(b, d_y, d_y + F, nullptr);
        if (rc == SVPF_OK && (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess))
            rc = SVPF_ERR_CUDA;
        float ms = 0.0f;
        if (rc == SVPF_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = SVPF_ERR_CUDA;
        if (rc == SVPF_OK && ms < best) {
            best = ms;
            best_t = t;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_y);
    svpf_batch_destroy(b);
    if (rc == SVPF_OK && best_t < 0) rc = SVPF_ERR_CUDA;
    if (rc == SVPF_OK) *best_tile = best_t;
    return rc;
}

}  // namespace

int svpf_autotune(const int* ns, int count, int ticks) {
    SVPF_TRACE();
    if (!ns || count < 1) return SVPF_ERR_INVALID_ARG;
    ticks = std::max(ticks, 1);
    for (int k = 0; k < count; ++k)
        if (ns[k] < 1 || ns[k] > SVPF_MAX_PARTICLES) return SVPF_ERR_INVALID_ARG;
    for (int k = 0; k < count; ++k) {
        int t = -1;
        const int rc = tune_one(ns[k], ticks, &t);
        if (rc != SVPF_OK) return rc;
        set_tuned_batch_tile(ns[k], t);
    }
    return SVPF_OK;
}

int svpf_batch_set_tile(svpf_batch_t* b, int f, int R, int S) {
    if (!b || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    int tile = -1;
    for (int t = kBatchTileLo; t <= kBatchTileHi; ++t)
        if (kTiles[t].R == R && kTiles[t].S == S) tile = t;
    if (tile < 0) return SVPF_ERR_INVALID_ARG;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return SVPF_ERR_CUDA;
    b->tiles[f] = (uint8_t)tile;
    drop_graph(b);
    return cudaMemcpy(b->d_tile + f, &b->tiles[f], 1, cudaMemcpyHostToDevice) == cudaSuccess ? SVPF_OK
                                                                                          : SVPF_ERR_CUDA;
}

int svpf_batch_tile_of_filter(const svpf_batch_t* b, int f, int* R, int* S) {
    if (!b || f < 0 || f >= b->F) return SVPF_ERR_INVALID_ARG;
    if (R) *R = kTiles[b->tiles[f]].R;
    if (S) *S = kTiles[b->tiles[f]].S;
    return SVPF_OK;
}

int svpf_tile_choice(int n, int* R, int* S) {
    int t = tuned_batch_tile(n);
    if (t < kBatchTileLo || t > kBatchTileHi) t = default_batch_tile(n);
    if (R) *R = kTiles[t].R;
    if (S) *S = kTiles[t].S;
    return SVPF_OK;
}

}  // extern "C"
