// C ABI of the solver context (include/nse2d.h, group 2). Written for this project.
#include <cstddef>
#include <string>
#include <cstring>
#include <vector>

#include "nse2d_internal.h"
#include "../../include/nse2d.h"

using namespace nse2d;


static Config to_config(const nse2d_config* a) {
    Config c;
    c.Nx = a->Nx; c.Ny = a->Ny; c.Lx = a->Lx; c.h = a->h; c.stretch = a->stretch; c.beta = a->beta;
    c.Ub = a->Ub; c.Reb = a->Reb; c.nu_override = a->nu_override; c.dt_init = a->dt_init; c.dt_max = a->dt_max;
    c.cfl = a->cfl; c.cvisc = a->cvisc; c.adapt = a->adapt; c.t_end = a->t_end; c.F0 = a->F0;
    c.nforce = a->nforce; c.lin_drag = a->lin_drag; c.free_slip = a->free_slip; c.mms = a->mms;
    c.mms_A0 = a->mms_A0; c.mms_eps = a->mms_eps; c.mms_Om = a->mms_Om; c.mms_kx = a->mms_kx;
    c.closure_diag = a->closure_diag; c.precision = a->precision;
    if (a->stretch == 2 && a->y_table) c.y_table.assign(a->y_table, a->y_table + (a->Ny > 0 ? a->Ny : 0));
    return c;
}

// precision 32: refresh the FP64 fields (and the stored rhs) from the split FP32 state
#define SYNC_FP64(ctx, with_rhs, s)                                                  \
    do {                                                                             \
        if ((ctx)->c->prec32 && export32((ctx)->c, (with_rhs), (s))) return -1;      \
    } while (0)

#define CHECK_CTX(ctx)                                    \
    do {                                                  \
        if (!(ctx) || !(ctx)->c) {                        \
            set_error("%s: null context", __func__);      \
            return -1;                                    \
        }                                                 \
    } while (0)

extern "C" {

void nse2d_config_default(nse2d_config* a) {
    const Config d;   // the reference defaults, src/common.cuh:42-114
    a->Nx = d.Nx; a->Ny = d.Ny; a->Lx = d.Lx; a->h = d.h; a->stretch = d.stretch; a->beta = d.beta;
    a->Ub = d.Ub; a->Reb = d.Reb; a->nu_override = d.nu_override; a->dt_init = d.dt_init; a->dt_max = d.dt_max;
    a->cfl = d.cfl; a->cvisc = d.cvisc; a->adapt = d.adapt; a->t_end = d.t_end; a->F0 = d.F0;
    a->nforce = d.nforce; a->lin_drag = d.lin_drag; a->free_slip = d.free_slip; a->mms = d.mms;
    a->mms_A0 = d.mms_A0; a->mms_eps = d.mms_eps; a->mms_Om = d.mms_Om; a->mms_kx = d.mms_kx;
    a->closure_diag = d.closure_diag; a->precision = d.precision;
    a->y_table = nullptr;
}

int nse2d_create(const nse2d_config* cfg, nse2d_ctx** out) {
    if (!cfg || !out) { set_error("nse2d_create: null argument"); return -1; }
    *out = nullptr;
    Context* c = nullptr;
    if (context_create(to_config(cfg), &c) != 0) return -1;
    *out = new nse2d_ctx{c};
    return 0;
}

int nse2d_destroy(nse2d_ctx* ctx) {
    if (!ctx) return 0;
    context_destroy(ctx->c);
    delete ctx;
    return 0;
}

int nse2d_set_omega(nse2d_ctx* ctx, const double* w, int where, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    NSE_CUDA_TRY(cudaMemcpyAsync(c->w, w, c->N * sizeof(double), where ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    return set_initial_omega(c, s);
}

int nse2d_set_state(nse2d_ctx* ctx, const double* w, const double* psi, int where, double t, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    const cudaMemcpyKind k = where ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    NSE_CUDA_TRY(cudaMemcpyAsync(c->w, w, c->N * sizeof(double), k, s));
    NSE_CUDA_TRY(cudaMemcpyAsync(c->psi, psi, c->N * sizeof(double), k, s));
    Ctl h{};
    h.t = t; h.dt = c->cfg.dt_init; h.next_out = 1e300; h.next_snap = 1e300; h.next_diag = 1e300;
    NSE_CUDA_TRY(cudaMemcpyAsync(c->ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    if (c->prec32 && split32(c, s)) return -1;
    if (refresh_maxima(c, s)) return -1;
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

int nse2d_get_fields(nse2d_ctx* ctx, double* w, double* psi, int where, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, false, s);
    Context* c = ctx->c;
    const cudaMemcpyKind k = where ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (w) NSE_CUDA_TRY(cudaMemcpyAsync(w, c->w, c->N * sizeof(double), k, s));
    if (psi) NSE_CUDA_TRY(cudaMemcpyAsync(psi, c->psi, c->N * sizeof(double), k, s));
    if (!where) NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

int nse2d_field_ptr(nse2d_ctx* ctx, int which, double** d_ptr) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    double* f[6] = {c->w, c->psi, c->w1, c->w2, c->rhs, c->J};
    if (which < 0 || which > 5 || !d_ptr) { set_error("nse2d_field_ptr: bad field %d", which); return -1; }
    *d_ptr = f[which];
    return 0;
}

int nse2d_get_field(nse2d_ctx* ctx, int which, double* host, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, which == 4, s);
    double* d = nullptr;
    if (nse2d_field_ptr(ctx, which, &d)) return -1;
    if (!host) { set_error("nse2d_get_field: null output"); return -1; }
    NSE_CUDA_TRY(cudaMemcpyAsync(host, d, ctx->c->N * sizeof(double), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

int nse2d_step(nse2d_ctx* ctx, int nsteps, int use_graph, cudaStream_t s) {
    CHECK_CTX(ctx);
    return run_steps(ctx->c, nsteps, use_graph != 0, s, false);
}

int nse2d_set_tridiag_form(nse2d_ctx* ctx, int clusters) {
    CHECK_CTX(ctx);
    return set_tridiag_form(ctx->c, clusters != 0);
}

int nse2d_step_store_rhs(nse2d_ctx* ctx, int nsteps, cudaStream_t s) {
    CHECK_CTX(ctx);
    return run_steps(ctx->c, nsteps, false, s, true);
}

int nse2d_step_timed(nse2d_ctx* ctx, int nsteps, double* kernel_ms, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    const int nk = launches_per_step(c);
    std::vector<cudaEvent_t> ev((size_t)nsteps * (nk + 1));
    for (auto& e : ev) NSE_CUDA_TRY(cudaEventCreate(&e));
    int rc = 0;
    for (int i = 0; i < nsteps && rc == 0; ++i) rc = enqueue_step_timed(c, s, &ev[(size_t)i * (nk + 1)]);
    if (rc == 0) {
        NSE_CUDA_TRY(cudaStreamSynchronize(s));
        for (int k = 0; k < nk; ++k) kernel_ms[k] = 0.0;
        for (int i = 0; i < nsteps; ++i)
            for (int k = 0; k < nk; ++k) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[(size_t)i * (nk + 1) + k], ev[(size_t)i * (nk + 1) + k + 1]);
                kernel_ms[k] += ms;
            }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

int nse2d_step_profiled(nse2d_ctx* ctx, double* step_ms, double* fft_ms, double* tridiag_ms, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    const int nk = launches_per_step(c);
    std::vector<cudaEvent_t> ev((size_t)nk + 1);
    for (auto& e : ev) NSE_CUDA_TRY(cudaEventCreate(&e));
    int rc = enqueue_step_timed(c, s, ev.data(), true);
    if (rc == 0) {
        NSE_CUDA_TRY(cudaStreamSynchronize(s));
        double tot = 0.0, fft = 0.0, tri = 0.0;
        for (int k = 0; k < nk; ++k) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            const std::string name = step_kernel_name(c, k);
            tot += ms;
            if (name.rfind("k_fft_fwd", 0) == 0 || name.rfind("k_ifft", 0) == 0) fft += ms;
            if (name.rfind("k_thomas", 0) == 0) tri += ms;
        }
        if (step_ms) *step_ms = tot;
        if (fft_ms) *fft_ms = fft;
        if (tridiag_ms) *tridiag_ms = tri;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

const char* nse2d_step_kernel_name(nse2d_ctx* ctx, int k) {
    if (!ctx || !ctx->c) return "";
    return step_kernel_name(ctx->c, k);
}

int nse2d_launches_per_step(nse2d_ctx* ctx) {
    CHECK_CTX(ctx);
    return launches_per_step(ctx->c);
}

int nse2d_set_dt(nse2d_ctx* ctx, double dt, cudaStream_t s) {
    CHECK_CTX(ctx);
    NSE_CUDA_TRY(cudaMemcpyAsync(&ctx->c->ctl->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

int nse2d_set_schedule(nse2d_ctx* ctx, double next_snap, double next_diag, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    double v[3] = {std::min(next_snap, next_diag), next_snap, next_diag};
    NSE_CUDA_TRY(cudaMemcpyAsync(&c->ctl->next_out, v, 3 * sizeof(double), cudaMemcpyHostToDevice, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

int nse2d_get_time(nse2d_ctx* ctx, double* t, double* dt, long long* step, double* umax3, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    NSE_CUDA_TRY(cudaMemcpyAsync(c->h_ctl, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    if (t) *t = c->h_ctl->t;
    if (dt) *dt = c->h_ctl->dt;
    if (step) *step = c->h_ctl->step;
    if (umax3) { umax3[0] = c->h_ctl->umax; umax3[1] = c->h_ctl->vmax; umax3[2] = c->h_ctl->vmaxm; }
    return 0;
}

int nse2d_run(nse2d_ctx* ctx, double next_snap, double next_diag, int stats_every, double t_end,
              long long max_steps, int* reason, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    if (max_steps <= 0) { set_error("nse2d_run: max_steps must be positive"); return -1; }
    if (stats_every < 0) { set_error("nse2d_run: stats_every must be >= 0"); return -1; }
    double sched[3] = {std::min(next_snap, next_diag), next_snap, next_diag};
    NSE_CUDA_TRY(cudaMemcpyAsync(&c->ctl->next_out, sched, 3 * sizeof(double), cudaMemcpyHostToDevice, s));
    // the run fields form the tail of the control block, from run to t_end
    Ctl* h = c->h_ctl;
    h->run = 1; h->halt = 0; h->halt_reason = 0; h->stats_every = stats_every;
    h->run_budget = max_steps; h->t_end = t_end;
    const size_t off = offsetof(Ctl, run), len = offsetof(Ctl, t_end) + sizeof(double) - off;
    NSE_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(c->ctl) + off, reinterpret_cast<char*>(h) + off, len,
                                 cudaMemcpyHostToDevice, s));
    if (run_until_halt(c, s)) return -1;
    NSE_CUDA_TRY(cudaMemcpyAsync(h, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    if (reason) *reason = h->halt_reason;
    const int zero = 0;
    NSE_CUDA_TRY(cudaMemcpyAsync(&c->ctl->run, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

int nse2d_row_moments(nse2d_ctx* ctx, double* out5, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, false, s);
    if (!out5) { set_error("nse2d_row_moments: null output"); return -1; }
    return row_moments(ctx->c, out5, s);
}

int nse2d_get_plan(nse2d_ctx* ctx, nse2d_plan* plan) {
    CHECK_CTX(ctx);
    if (!plan) { set_error("nse2d_get_plan: null plan"); return -1; }
    const PlanForms f = get_plan(ctx->c);
    plan->stage_tma = f.stage_tma ? 1 : 0;
    plan->tridiag_clusters = f.clusters ? 1 : 0;
    plan->rowfft_prefetch = f.rowfft_pf ? 1 : 0;
    plan->max_fused = f.max_fused ? 1 : 0;
    plan->pdl = f.pdl ? 1 : 0;
    return 0;
}

int nse2d_set_plan(nse2d_ctx* ctx, const nse2d_plan* plan) {
    CHECK_CTX(ctx);
    if (!plan) { set_error("nse2d_set_plan: null plan"); return -1; }
    return set_plan(ctx->c, PlanForms{plan->stage_tma != 0, plan->tridiag_clusters != 0, plan->rowfft_prefetch != 0,
                                      plan->max_fused != 0, plan->pdl != 0});
}

// Every plan the context can use, timed over trial_steps graph-replayed steps from the current
// state; the state (fields and control block) is saved before and restored after, so only the
// plan changes. The fastest plan stays set.
int nse2d_autotune_plan(nse2d_ctx* ctx, int trial_steps, nse2d_plan* best, double* ms_per_step, cudaStream_t s) {
    CHECK_CTX(ctx);
    if (trial_steps <= 0) { set_error("nse2d_autotune_plan: trial_steps must be positive"); return -1; }
    Context* c = ctx->c;
    const size_t fb = c->N * (c->prec32 ? sizeof(float) : sizeof(double));
    void* wsrc = c->prec32 ? (void*)c->wf : (void*)c->w;
    void* psrc = c->prec32 ? (void*)c->psif : (void*)c->psi;
    void *wsave = nullptr, *psave = nullptr;
    Ctl saved{};
    NSE_CUDA_TRY(cudaMalloc(&wsave, fb));
    if (cudaMalloc(&psave, fb) != cudaSuccess) { cudaFree(wsave); set_error("nse2d_autotune_plan: out of memory"); return -1; }
    cudaEvent_t a = nullptr, b = nullptr;
    int rc = 0;
    double best_ms = 1e300;
    nse2d_plan bp{};
    auto save = [&]() -> int {
        NSE_CUDA_TRY(cudaMemcpyAsync(wsave, wsrc, fb, cudaMemcpyDeviceToDevice, s));
        NSE_CUDA_TRY(cudaMemcpyAsync(psave, psrc, fb, cudaMemcpyDeviceToDevice, s));
        NSE_CUDA_TRY(cudaMemcpyAsync(&saved, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
        NSE_CUDA_TRY(cudaStreamSynchronize(s));
        return 0;
    };
    auto restore = [&]() -> int {
        NSE_CUDA_TRY(cudaMemcpyAsync(wsrc, wsave, fb, cudaMemcpyDeviceToDevice, s));
        NSE_CUDA_TRY(cudaMemcpyAsync(psrc, psave, fb, cudaMemcpyDeviceToDevice, s));
        NSE_CUDA_TRY(cudaMemcpyAsync(c->ctl, &saved, sizeof(Ctl), cudaMemcpyHostToDevice, s));
        NSE_CUDA_TRY(cudaStreamSynchronize(s));
        return 0;
    };
    const bool st_ok = c->prec32 ? c->stage32_tma_ok : c->stage_tma_ok;
    const bool mf_ok = c->rowfft_pf_ok && c->cfg.adapt && !c->prec32;   // the fused max needs the prefetching form
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) { set_error("event"); rc = -1; }
    if (rc == 0) rc = save();
    for (int st = st_ok ? 1 : 0; rc == 0 && st >= 0; --st)
        for (int cl = c->thomas_cluster_ok ? 1 : 0; rc == 0 && cl >= 0; --cl)
            for (int pf = c->rowfft_pf_ok ? 1 : 0; rc == 0 && pf >= 0; --pf)
                for (int mf = (pf && mf_ok) ? 1 : 0; rc == 0 && mf >= 0; --mf)
                for (int pd = 1; rc == 0 && pd >= 0; --pd) {
                    if ((rc = set_plan(c, PlanForms{st != 0, cl != 0, pf != 0, mf != 0, pd != 0}))) break;
                    if ((rc = run_steps(c, 1, true, s, false))) break;           // capture and warm
                    cudaEventRecord(a, s);
                    if ((rc = run_steps(c, trial_steps, true, s, false))) break;
                    cudaEventRecord(b, s);
                    if (cudaEventSynchronize(b) != cudaSuccess) {
                        set_error("nse2d_autotune_plan: %s", cudaGetErrorString(cudaGetLastError()));
                        rc = -1;
                        break;
                    }
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, a, b);
                    if (ms / trial_steps < best_ms) { best_ms = ms / trial_steps; bp = nse2d_plan{st, cl, pf, mf, pd}; }
                    if ((rc = restore())) break;
                }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (rc == 0) rc = restore();
    cudaFree(wsave);
    cudaFree(psave);
    if (rc) return rc;
    if (best) *best = bp;
    if (ms_per_step) *ms_per_step = best_ms;
    return set_plan(c, PlanForms{bp.stage_tma != 0, bp.tridiag_clusters != 0, bp.rowfft_prefetch != 0, bp.max_fused != 0,
                                 bp.pdl != 0});
}

int nse2d_stats_device(nse2d_ctx* ctx, int every, cudaStream_t s) {
    CHECK_CTX(ctx);
    return stats_device(ctx->c, every, s);
}

int nse2d_stats_read(nse2d_ctx* ctx, double* out5, double* T, cudaStream_t s) {
    CHECK_CTX(ctx);
    return stats_read(ctx->c, out5, T, s);
}

int nse2d_spectra_accumulate(nse2d_ctx* ctx, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, false, s);
    return spectra_accumulate(ctx->c, s);
}

int nse2d_spectra(nse2d_ctx* ctx, double* kx, double* Eu, double* Ev, int* samples, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    const int H = c->H;
    std::vector<double> acc(2 * (size_t)c->Hp, 0.0);
    if (c->spec_acc) {
        NSE_CUDA_TRY(cudaMemcpyAsync(acc.data(), c->spec_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        NSE_CUDA_TRY(cudaStreamSynchronize(s));
    }
    const int n = c->spec_samples;
    for (int k = 0; k < H; ++k) {
        if (kx) kx[k] = (2.0 * 3.141592653589793 * (double)k) / c->cfg.Lx;   // fill_kx_array_kernel, diag.cu:868-873
        double eu = acc[k], ev = acc[(size_t)c->Hp + k];
        if (n > 0) { eu /= n; ev /= n; }
        if (Eu) Eu[k] = eu;
        if (Ev) Ev[k] = ev;
    }
    if (samples) *samples = n;
    return 0;
}

int nse2d_nonfinite(nse2d_ctx* ctx, int* flag, cudaStream_t s) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    NSE_CUDA_TRY(cudaMemcpyAsync(c->h_ctl, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    *flag = c->h_ctl->nonfinite;
    return 0;
}

int nse2d_poisson_solve(nse2d_ctx* ctx, const double* d_w, double* d_psi, cudaStream_t s) {
    CHECK_CTX(ctx);
    return poisson_solve(ctx->c, d_w, d_psi, s);
}

int nse2d_max_uv(nse2d_ctx* ctx, double* out3, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, false, s);
    Context* c = ctx->c;
    if (launch_maxuv(c, c->psi, false, s)) return -1;
    return nse2d_get_time(ctx, nullptr, nullptr, nullptr, out3, s);
}

int nse2d_diagnostics(nse2d_ctx* ctx, int t0_row, double* out29, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, t0_row == 0, s);
    return diagnostics_row(ctx->c, t0_row, out29, s);
}

int nse2d_rhs_at_state(nse2d_ctx* ctx, double t, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, false, s);
    Context* c = ctx->c;
    if (rhs_at_state(c, c->w, c->psi, c->J, c->rhs, t, s)) return -1;
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

int nse2d_uv(nse2d_ctx* ctx, double* d_u, double* d_v, cudaStream_t s) {
    CHECK_CTX(ctx);
    SYNC_FP64(ctx, false, s);
    return uv_from_psi(ctx->c, ctx->c->psi, d_u, d_v, s);
}

int nse2d_metrics(nse2d_ctx* ctx, int which, double* out) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    const std::vector<double>* v[5] = {&c->h_y, &c->h_a_node, &c->h_a_edge, &c->h_dy_edge, &c->h_w_node};
    if (which < 0 || which > 4 || !out) { set_error("nse2d_metrics: bad metric %d", which); return -1; }
    std::memcpy(out, v[which]->data(), v[which]->size() * sizeof(double));
    return 0;
}

int nse2d_scalar(nse2d_ctx* ctx, int which, double* out) {
    CHECK_CTX(ctx);
    Context* c = ctx->c;
    const double v[7] = {c->nu, c->dx, c->deta, c->invA_full, c->meanFx_A, c->psi_bot, c->psi_top};
    if (which < 0 || which > 6 || !out) { set_error("nse2d_scalar: bad index %d", which); return -1; }
    *out = v[which];
    return 0;
}

const char* nse2d_last_error(void) { return get_error(); }

}  // extern "C"
