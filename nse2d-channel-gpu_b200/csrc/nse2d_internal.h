// Internal interface between the C-ABI layer and the solver implementation.
#pragma once
#include <utility>

#include "common.cuh"

namespace nse2d {
// A step kernel (each begins with pdl_begin), with the programmatic-serialisation attribute when
// the plan asks for it; extra: another launch attribute (the cluster shape), or nullptr.
template <typename... KArgs, typename... Args>
inline int launch_step_kernel(const Context* c, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, const cudaLaunchAttribute* extra, Args&&... args) {
    cudaLaunchConfig_t lc{};
    cudaLaunchAttribute at[2];
    unsigned na = 0;
    if (extra) at[na++] = *extra;
    if (c->pdl) {
        at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    lc.gridDim = grid; lc.blockDim = block; lc.dynamicSmemBytes = smem; lc.stream = s;
    lc.attrs = at; lc.numAttrs = na;
    NSE_CUDA_TRY(cudaLaunchKernelEx(&lc, kern, std::forward<Args>(args)...));
    return 0;
}

int build_y_metrics(const Config& c, std::vector<double>& y, std::vector<double>& a_node,
                    std::vector<double>& a_edge, std::vector<double>& dy_edge, std::vector<double>& w_node);
int context_create(const Config& cfg, Context** out);
void context_destroy(Context* c);
int launch_stage(Context* c, int stage, const double* w_in, const double* w_n, double* w_out, cudaStream_t s,
                 double* rhs_out = nullptr);
int launch_fft_fwd(Context* c, const double* src, cudaStream_t s);
int launch_thomas(Context* c, cudaStream_t s);
int launch_thomas_maps(Context* c, cudaStream_t s, bool homog = false);
int launch_thomas_apply(Context* c, cudaStream_t s, bool homog = false);
int launch_thomas_cluster(Context* c, cudaStream_t s, bool homog = false);
// learned closure (closure.cu)
struct Cnn;
int cnn_forward(Cnn* n, const double* w, const double* psi, const double* u, const double* v, double* tau, cudaStream_t s);
bool cnn_matches(const Cnn* n, int Nx, int Ny);
int thomas_launches(const Context* c);
const char* thomas_kernel_name(const Context* c, int i);
int launch_thomas_part(Context* c, int i, cudaStream_t s, bool homog = false);
// FP32-bulk variant (csrc/solver32.cu)
int setup32(Context* c);
// Select the cluster (clusters != 0, where available) or the two-pass tridiagonal solve; drops
// the context's captured step graphs when the form changes (solver.cu).
int set_tridiag_form(Context* c, bool clusters);
// the kernel forms of a context's step (nse2d_plan)
struct PlanForms { bool stage_tma, clusters, rowfft_pf, max_fused, pdl; };
PlanForms get_plan(const Context* c);
int set_plan(Context* c, const PlanForms& f);
int refresh_maxima(Context* c, cudaStream_t s);
// 2-D tensor map of a [Ny][Nx] FP64 (or FP32) field with a bw x bh box (solver.cu).
int encode_map_2d(CUtensorMap* map, const void* base, bool f32, int Nx, int Ny, int bw, int bh);
void destroy32(Context* c);
int split32(Context* c, cudaStream_t s);
int export32(Context* c, bool with_rhs, cudaStream_t s);
int step32_impl(Context* c, cudaStream_t s, bool store_rhs, cudaEvent_t* ev);
const char* step32_kernel_name(const Context* c, int k);
int launch_ifft_thom(Context* c, double* psi, double* w, int stage, bool do_thom, bool closure, cudaStream_t s,
                     bool advance = false);
int launch_thom(Context* c, double* w, const double* psi, cudaStream_t s);
int launch_maxuv(Context* c, const double* psi, bool set_dt, cudaStream_t s, bool next_only = false);
int poisson_solve(Context* c, const double* w, double* psi, cudaStream_t s);
int enqueue_step(Context* c, cudaStream_t s, bool store_rhs);
int launches_per_step(const Context* c);
int enqueue_step_timed(Context* c, cudaStream_t s, cudaEvent_t* ev, bool store_rhs = false);
const char* step_kernel_name(const Context* c, int k);
int run_steps(Context* c, int nsteps, bool use_graph, cudaStream_t s, bool store_rhs);
int set_initial_omega(Context* c, cudaStream_t s);
int diagnostics_row(Context* c, int t0_row, double* out29, cudaStream_t s);
int rhs_at_state(Context* c, const double* w, const double* psi, double* J, double* rhs, double tm, cudaStream_t s);
int uv_from_psi(Context* c, const double* psi, double* u, double* v, cudaStream_t s);
int launch_fft_all_rows(Context* c, const double* src, cudaStream_t s);
int run_until_halt(Context* c, cudaStream_t s);
int row_moments(Context* c, double* out5, cudaStream_t s);
int spectra_accumulate(Context* c, cudaStream_t s);
int enqueue_stats(Context* c, cudaStream_t s);
int stats_device(Context* c, int every, cudaStream_t s);
int stats_read(Context* c, double* out5, double* T, cudaStream_t s);
int spectra_accumulate_uv(Context* c, const double* u, const double* v, cudaStream_t s);
// after a launch of the reference-compatible operators (ops.cu): keep a CUDA error for
// nse2d_last_error and, unless nse2d_set_abort_on_error(0), print it and abort as the reference does
void compat_check_launch(const char* what);
bool compat_free_slip();
}  // namespace nse2d

// The C ABI's handle: one solver context.
struct nse2d_ctx {
    nse2d::Context* c;
};
