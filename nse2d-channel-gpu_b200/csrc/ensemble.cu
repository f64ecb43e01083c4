// Batched ensembles: many independent channels (each its own solver context, grid, physics and
// adaptive dt) advanced together by ONE graph launch. Written for this project; the reference
// runs one channel per process.
//
// The graph holds a WHILE node whose body is one step of every member: the members are dealt
// round-robin onto G branches (streams forked from the capture stream and joined back), each
// branch running its members' captured steps one after the other, so up to G members' kernels
// share the GPU at a time; a last kernel counts the steps down and ends the loop. Small
// channels cannot fill a B200 alone, and 64 of them launched one after the other spend most of
// their time in launch gaps; concurrent branches fill the machine. The best G depends on the
// member sizes and is chosen by nse2d_ensemble_autotune, which times every candidate. Members
// are independent, so G never changes a result.
#include <algorithm>
#include <vector>

#include "nse2d_internal.h"
#include "../../include/nse2d.h"

namespace nse2d {
namespace {

__global__ void k_ensemble_cond(int* count, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    *count -= 1;
    cudaGraphSetConditional(h, *count > 0 ? 1u : 0u);
}

struct Ensemble {
    std::vector<Context*> m;
    int groups = 0;
    int* d_count = nullptr;
    cudaStream_t cap = nullptr;
    std::vector<cudaStream_t> branch;
    cudaGraphExec_t exec = nullptr;
};

int ensemble_build(Ensemble* e, int groups, bool force = false) {
    const int n = (int)e->m.size();
    groups = std::max(1, std::min(groups, n));
    if (e->exec && e->groups == groups && !force) return 0;
    if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
    while ((int)e->branch.size() < groups) {
        cudaStream_t s;
        NSE_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        e->branch.push_back(s);
    }
    cudaGraph_t g = nullptr;
    NSE_CUDA_TRY(cudaGraphCreate(&g, 0));
    std::vector<cudaEvent_t> ev;
    auto done = [&](int rc) {
        for (auto x : ev) cudaEventDestroy(x);
        if (g) cudaGraphDestroy(g);
        return rc;
    };
    cudaGraphConditionalHandle h;
    cudaError_t err = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (err != cudaSuccess) { set_error("ensemble graph: %s", cudaGetErrorString(err)); return done(-1); }
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    err = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    if (err != cudaSuccess) { set_error("ensemble graph: %s", cudaGetErrorString(err)); return done(-1); }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    ev.resize(1 + groups);
    for (auto& x : ev) NSE_CUDA_TRY(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    err = cudaStreamBeginCaptureToGraph(e->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) { set_error("ensemble capture: %s", cudaGetErrorString(err)); return done(-1); }
    int rc = 0;
    cudaEventRecord(ev[0], e->cap);                                   // fork
    for (int b = 0; b < groups && rc == 0; ++b) {
        cudaStreamWaitEvent(e->branch[b], ev[0], 0);
        for (int i = b; i < n && rc == 0; i += groups) rc = enqueue_step(e->m[i], e->branch[b], false);
        cudaEventRecord(ev[1 + b], e->branch[b]);                     // join
        cudaStreamWaitEvent(e->cap, ev[1 + b], 0);
    }
    if (rc == 0) k_ensemble_cond<<<1, 32, 0, e->cap>>>(e->d_count, h);
    cudaGraph_t captured = nullptr;
    err = cudaStreamEndCapture(e->cap, &captured);
    if (rc != 0) return done(-1);
    if (err != cudaSuccess) { set_error("ensemble capture: %s", cudaGetErrorString(err)); return done(-1); }
    err = cudaGraphInstantiate(&e->exec, g, 0);
    if (err != cudaSuccess) { set_error("ensemble instantiate: %s", cudaGetErrorString(err)); return done(-1); }
    e->groups = groups;
    return done(0);
}

int ensemble_step(Ensemble* e, int nsteps, cudaStream_t s) {
    if (nsteps <= 0) return 0;
    if (!e->exec && ensemble_build(e, e->groups > 0 ? e->groups : (int)e->m.size())) return -1;
    NSE_CUDA_TRY(cudaMemcpyAsync(e->d_count, &nsteps, sizeof(int), cudaMemcpyHostToDevice, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));     // nsteps lives on this stack frame
    NSE_CUDA_TRY(cudaGraphLaunch(e->exec, s));
    return 0;
}

}  // namespace
}  // namespace nse2d

using namespace nse2d;

struct nse2d_ensemble {
    Ensemble e;
};

extern "C" {

int nse2d_ensemble_autotune(nse2d_ensemble* en, int trial_steps, int* groups_out, double* ms_per_step_out,
                            cudaStream_t s);

int nse2d_ensemble_create(nse2d_ctx* const* members, int n, nse2d_ensemble** out) {
    if (!members || n <= 0 || !out) { set_error("nse2d_ensemble_create: bad arguments"); return -1; }
    *out = nullptr;
    auto* en = new nse2d_ensemble();
    for (int i = 0; i < n; ++i) {
        if (!members[i] || !members[i]->c) { delete en; set_error("nse2d_ensemble_create: member %d is null", i); return -1; }
        for (int k = 0; k < i; ++k)
            if (members[k]->c == members[i]->c) { delete en; set_error("nse2d_ensemble_create: member %d repeated", i); return -1; }
        en->e.m.push_back(members[i]->c);
    }
    // Members take the two-pass tridiagonal solve: its plain grids share the SMs with the other
    // branches' kernels, while the cluster form's persistent clusters, sized to fill the device,
    // serialise the branches (64-channel workload: 1.33 against 1.92 ms per ensemble step).
    for (Context* c : en->e.m)
        if (set_tridiag_form(c, false)) { delete en; return -1; }
    if (cudaMalloc((void**)&en->e.d_count, sizeof(int)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&en->e.cap, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("nse2d_ensemble_create: %s", cudaGetErrorString(cudaGetLastError()));
        if (en->e.d_count) cudaFree(en->e.d_count);
        delete en;
        return -1;
    }
    en->e.groups = n;
    *out = en;
    return 0;
}

int nse2d_ensemble_destroy(nse2d_ensemble* en) {
    if (!en) return 0;
    Ensemble& e = en->e;
    if (e.exec) cudaGraphExecDestroy(e.exec);
    for (auto s : e.branch) cudaStreamDestroy(s);
    if (e.cap) cudaStreamDestroy(e.cap);
    if (e.d_count) cudaFree(e.d_count);
    delete en;
    return 0;
}

int nse2d_ensemble_set_groups(nse2d_ensemble* en, int groups) {
    if (!en) { set_error("nse2d_ensemble_set_groups: null ensemble"); return -1; }
    return ensemble_build(&en->e, groups);
}

int nse2d_ensemble_step(nse2d_ensemble* en, int nsteps, cudaStream_t s) {
    if (!en) { set_error("nse2d_ensemble_step: null ensemble"); return -1; }
    return ensemble_step(&en->e, nsteps, s);
}

// Coordinate descent over the kernel plans of the members: for every class of members with the
// same grid and precision, each form the class can switch (stage kernel, tridiagonal form, row
// transform form) is toggled for the whole class, the ensemble graph rebuilt and one ensemble
// step timed; a toggle that is not faster is undone. Then the branch count is tuned again.
int nse2d_ensemble_autotune_plans(nse2d_ensemble* en, int trial_steps, int* groups_out, double* ms_per_step_out,
                                  cudaStream_t s) {
    if (!en || trial_steps <= 0) { set_error("nse2d_ensemble_autotune_plans: bad arguments"); return -1; }
    Ensemble& e = en->e;
    int g0 = 0;
    double ms0 = 0.0;
    if (nse2d_ensemble_autotune(en, trial_steps, &g0, &ms0, s)) return -1;
    cudaEvent_t a, b;
    NSE_CUDA_TRY(cudaEventCreate(&a));
    NSE_CUDA_TRY(cudaEventCreate(&b));
    auto time_step = [&](double& ms) -> int {
        if (ensemble_build(&e, e.groups, true) || ensemble_step(&e, 1, s)) return -1;
        cudaEventRecord(a, s);
        if (ensemble_step(&e, trial_steps, s)) return -1;
        cudaEventRecord(b, s);
        NSE_CUDA_TRY(cudaEventSynchronize(b));
        float f = 0.f;
        cudaEventElapsedTime(&f, a, b);
        ms = f / trial_steps;
        return 0;
    };
    struct Cls { int Nx, Ny; bool p32; std::vector<Context*> m; };
    std::vector<Cls> cls;
    for (Context* c : e.m) {
        auto it = std::find_if(cls.begin(), cls.end(),
                               [&](const Cls& k) { return k.Nx == c->Nx && k.Ny == c->Ny && k.p32 == c->prec32; });
        if (it == cls.end()) { cls.push_back({c->Nx, c->Ny, c->prec32, {}}); it = cls.end() - 1; }
        it->m.push_back(c);
    }
    auto plan_of = [](const Context* c, bool* v) {
        const PlanForms f = get_plan(c);
        v[0] = f.stage_tma; v[1] = f.clusters; v[2] = f.rowfft_pf; v[3] = f.max_fused; v[4] = f.pdl;
    };
    double best = 0.0;
    int rc = time_step(best);
    for (size_t k = 0; rc == 0 && k < cls.size(); ++k) {
        Context* c0 = cls[k].m[0];
        const bool ok[5] = {c0->prec32 ? c0->stage32_tma_ok : c0->stage_tma_ok, c0->thomas_cluster_ok, c0->rowfft_pf_ok,
                            c0->rowfft_pf_ok && c0->cfg.adapt && !c0->prec32, true};
        for (int f = 0; rc == 0 && f < 5; ++f) {
            if (!ok[f]) continue;
            bool v[5];
            plan_of(c0, v);
            v[f] = !v[f];
            for (Context* c : cls[k].m)
                if ((rc = set_plan(c, PlanForms{v[0], v[1], v[2], v[3], v[4]}))) break;
            double ms = 0.0;
            if (rc == 0) rc = time_step(ms);
            if (rc == 0 && !(ms < best)) {                       // not faster: undo
                v[f] = !v[f];
                for (Context* c : cls[k].m)
                    if ((rc = set_plan(c, PlanForms{v[0], v[1], v[2], v[3], v[4]}))) break;
            } else if (rc == 0) {
                best = ms;
            }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (ensemble_build(&e, e.groups, true)) return -1;
    return nse2d_ensemble_autotune(en, trial_steps, groups_out, ms_per_step_out, s);
}

int nse2d_ensemble_autotune(nse2d_ensemble* en, int trial_steps, int* groups_out, double* ms_per_step_out,
                            cudaStream_t s) {
    if (!en || trial_steps <= 0) { set_error("nse2d_ensemble_autotune: bad arguments"); return -1; }
    Ensemble& e = en->e;
    const int n = (int)e.m.size();
    std::vector<int> cand;
    for (int g = 1; g < n; g *= 2) cand.push_back(g);
    cand.push_back(n);
    cudaEvent_t a, b;
    NSE_CUDA_TRY(cudaEventCreate(&a));
    NSE_CUDA_TRY(cudaEventCreate(&b));
    int best = n;
    double best_ms = 1e300;
    int rc = 0;
    for (int g : cand) {
        if ((rc = ensemble_build(&e, g, true))) break;
        if ((rc = ensemble_step(&e, 1, s))) break;                    // warm: first launch of this graph
        cudaEventRecord(a, s);
        if ((rc = ensemble_step(&e, trial_steps, s))) break;
        cudaEventRecord(b, s);
        if (cudaEventSynchronize(b) != cudaSuccess) { set_error("autotune: %s", cudaGetErrorString(cudaGetLastError())); rc = -1; break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms / trial_steps < best_ms) { best_ms = ms / trial_steps; best = g; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (groups_out) *groups_out = best;
    if (ms_per_step_out) *ms_per_step_out = best_ms;
    return ensemble_build(&e, best, true);
}

}  // extern "C"
