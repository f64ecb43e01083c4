/*
 * nse2d-b200: C ABI of the B200 channel time step (libnse2d_b200.so).
 *
 * Two groups of entry points:
 *
 * 1. The C-linkage operator launchers of the reference, same names, same argument order
 *    and meaning, asynchronous on the given stream, all pointers device memory owned by
 *    the caller (reference: src/test_api.cu:8-92, built there with -DEXPORT_TEST_API).
 *    Like the reference they return nothing; on a CUDA error they print the error and
 *    abort the process (src/common.cuh:116-117), unless nse2d_set_abort_on_error(0) was
 *    called, in which case the error is kept for nse2d_last_error().
 *
 * 2. nse2d_* entry points with an int status (0 = success, nonzero = error, message in
 *    nse2d_last_error()). They drive the whole SSPRK(3,3) time step of the reference's
 *    time loop (src/main.cu:434-541) on a solver context that owns its fields and
 *    workspace; they replace the reference's C++ driver-side calls (Poisson2D_Z2Z in
 *    src/poisson.cuh:18-119, the launch_* functions of src/ops.cuh and src/diag.cuh).
 *
 * Arrays are row-major [Ny][Nx] FP64 (x fastest), metrics [Ny] / [Ny-1], as in the
 * reference (src/common.cuh:127-130).
 */
#ifndef NSE2D_B200_H
#define NSE2D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* cudaStream_t;

/* ---------------------------------------------------------------------------------------
 * 1. Reference test API (src/test_api.cu)
 * ------------------------------------------------------------------------------------- */
/* u = a psi_eta / (2 deta), v = -psi_x / (2 dx), clamped at the walls. test_api.cu:8-18 */
void testapi_uv_from_psi_mapped(const double* d_psi, double* d_u, double* d_v, int Nx, int Ny,
                                double inv_dx, double inv_deta, const double* d_a_node,
                                cudaStream_t s);
/* omega = -(dxx psi + mapped dyy psi) on interior rows. test_api.cu:20-30 */
void testapi_omega_from_psi_interior_mapped(double* d_w, const double* d_psi, int Nx, int Ny,
                                            double inv_dx2, double inv_deta2,
                                            const double* d_a_node, const double* d_a_edge,
                                            cudaStream_t s);
/* Thom wall vorticity (no-slip; zero with nse2d_testapi_set_free_slip(1)). test_api.cu:32-42 */
void testapi_thom_wall_vorticity_mapped(double* d_w, const double* d_psi, int Nx, int Ny,
                                        const double* d_dy_edge, double psi_bot, double psi_top,
                                        cudaStream_t s);
/* mapped Arakawa Jacobian u.grad(omega) = -(J1+J2+J3)/3, walls 0. test_api.cu:44-53 */
void testapi_arakawa_J_mapped(const double* d_psi, const double* d_w, double* d_J, int Nx, int Ny,
                              double inv_dx, double inv_deta, const double* d_a_node,
                              cudaStream_t s);
/* advective reference u omega_x + v omega_y from (u, v). test_api.cu:55-65 */
void testapi_compute_adv_from_uv_mapped(const double* d_u, const double* d_v, const double* d_omg,
                                        double* d_Jref, int Nx, int Ny, double inv_dx,
                                        double inv_deta, const double* d_a_node, cudaStream_t s);
/* conservative flux form. test_api.cu:67-77 */
void testapi_compute_adv_flux_mapped(const double* d_u, const double* d_v, const double* d_omg,
                                     double* d_Jref, int Nx, int Ny, double inv_dx,
                                     double inv_deta, const double* d_a_node, cudaStream_t s);
/* J1, J2, J3 and Jadv separately; any output may be NULL. test_api.cu:79-92 */
void testapi_arakawa_J_mapped_split(const double* d_psi, const double* d_omg, double* d_J1,
                                    double* d_J2, double* d_J3, double* d_Jadv, int Nx, int Ny,
                                    double inv_dx, double inv_deta, const double* d_a_node,
                                    cudaStream_t s);

/* Behaviour switches of group 1 (no counterpart in the reference, which fixes both at
 * compile time: CUDA_CHECK aborts, FREE_SLIP_WALLS selects the wall closure). */
void nse2d_set_abort_on_error(int on);
void nse2d_testapi_set_free_slip(int on);

/* ---------------------------------------------------------------------------------------
 * 2. Solver context API
 * ------------------------------------------------------------------------------------- */
/* The reference's Grid + Params fields used by the time step (src/common.cuh:42-114),
 * with the reference defaults from nse2d_config_default(). */
typedef struct nse2d_config {
    int    Nx, Ny;            /* Nx a power of two >= 4; Ny >= 5 */
    double Lx, h;
    int    stretch;           /* 0 = none (uniform), 1 = tanh (src/grid.cu:33-45), 2 = table
                                 (y_table, src/grid.cu:46-78) */
    double beta;
    double Ub, Reb, nu_override;   /* nu = nu_override if >= 0, else 2 h Ub / Reb */
    double dt_init, dt_max, cfl, cvisc;
    int    adapt;             /* adaptive dt (src/main.cu:439-464) */
    double t_end, F0;
    int    nforce;
    double lin_drag;
    int    free_slip;         /* free-slip walls (omega_wall = 0) instead of Thom */
    int    mms;
    double mms_A0, mms_eps, mms_Om;
    int    mms_kx;
    int    closure_diag;      /* accumulate the wall-update enstrophy (Jwall columns) */
    int    precision;         /* 64 (FP64 throughout) or 32 (FP32 bulk with FP64 islands: the
                                 x-mean base profiles and the tridiagonal solve's arithmetic and
                                 table, over an FP32 spectral buffer; no MMS forcing, no closure
                                 diagnostics). With 32, the
                                 FP64 fields behind nse2d_field_ptr are refreshed only by the
                                 calls that read them (fields, diagnostics, uv, statistics). */
    const double* y_table;    /* stretch 2: the Ny node coordinates y_0 < ... < y_{Ny-1} (host
                                 array, copied by nse2d_create; NULL otherwise) */
} nse2d_config;

typedef struct nse2d_ctx nse2d_ctx;

void nse2d_config_default(nse2d_config* cfg);
int  nse2d_create(const nse2d_config* cfg, nse2d_ctx** out);
int  nse2d_destroy(nse2d_ctx* ctx);

/* Set omega (where = 0: host array, 1: device array), then the initial Poisson solve and
 * Thom closure; t = 0, dt = dt_init (src/main.cu:197-215). Synchronous. */
int  nse2d_set_omega(nse2d_ctx* ctx, const double* w, int where, cudaStream_t s);
/* Set omega and psi as they are (resume), and the time t. Synchronous. */
int  nse2d_set_state(nse2d_ctx* ctx, const double* w, const double* psi, int where, double t,
                     cudaStream_t s);
/* Copy omega and/or psi out (either may be NULL). where = 0: host (synchronous), 1: device. */
int  nse2d_get_fields(nse2d_ctx* ctx, double* w, double* psi, int where, cudaStream_t s);
/* Device pointer of a context field: 0 omega, 1 psi, 2 omega1, 3 omega2, 4 rhs, 5 J. */
int  nse2d_field_ptr(nse2d_ctx* ctx, int which, double** d_ptr);
/* Copy context field `which` (numbered as for nse2d_field_ptr) to a host array. Synchronous. */
int  nse2d_get_field(nse2d_ctx* ctx, int which, double* host, cudaStream_t s);

/* Advance nsteps SSPRK(3,3) steps, asynchronously. With adapt, dt is computed on the
 * device before every step (max |u|, |v|, |v| a, CFL and viscous limits, trimming to
 * the next output time); otherwise the dt of nse2d_set_dt / dt_init is used. use_graph:
 * replay one captured CUDA graph per step. */
int  nse2d_step(nse2d_ctx* ctx, int nsteps, int use_graph, cudaStream_t s);
/* The tridiagonal solve of the Poisson step: clusters != 0 selects the one-pass form on
 * persistent thread-block clusters (the default where it can be resident: fastest for a
 * channel that has the device to itself), 0 the two-pass form on plain grids (which shares
 * the device with concurrent work). Both give the reference's solve to round-off, not the
 * same bits. Synchronises the device when the form changes (the step graph is captured
 * again). */
int  nse2d_set_tridiag_form(nse2d_ctx* ctx, int clusters);
/* The kernel forms of a context's step (no counterpart in the reference, which has one form of
 * each operator): stage_tma, the persistent stage kernel fed by TMA boxes (1) or the one with a
 * CTA per tile and plain halo loads (0; grids with Nx < 128, or Nx < 256 in precision 32, have
 * only this one); tridiag_clusters, as nse2d_set_tridiag_form; rowfft_prefetch, the row
 * transforms whose rows are prefetched into shared memory by bulk copies (1; Nx = 4096 in
 * precision 64 only) or read by plain loads (0); max_fused, with the prefetching transforms in an
 * adaptive FP64 step, the max reduction of psi inside the stage-3 inverse transform and dt
 * computed by the next step's stage kernel (1) or a separate max reduction at the start of the
 * step (0, the default: the faster at 4096x2049); pdl, the step kernels launched with
 * programmatic dependent launch (1: a kernel's launch is processed while the one before it
 * finishes, and its CTAs wait on the device for that one's completion before they read or write
 * anything) or in plain stream order (0, the default). Every form gives
 * the same step to round-off (the two stage forms, the two max forms and the two launch forms
 * to the bit). nse2d_set_plan falls back to the form a context can use and synchronises the
 * device when a form changes (the step graphs are captured again); nse2d_get_plan reports the
 * forms in use (max_fused as it takes effect). */
typedef struct nse2d_plan {
    int stage_tma, tridiag_clusters, rowfft_prefetch, max_fused, pdl;
} nse2d_plan;
int  nse2d_get_plan(nse2d_ctx* ctx, nse2d_plan* plan);
int  nse2d_set_plan(nse2d_ctx* ctx, const nse2d_plan* plan);
/* Times every plan the context can use over trial_steps graph-replayed steps from the current state
 * and keeps the fastest (best and its ms per step are reported; either may be NULL). The fields
 * and the control block are saved before and restored after, so only the plan changes; two
 * temporary fields are allocated for that. Synchronous. */
int  nse2d_autotune_plan(nse2d_ctx* ctx, int trial_steps, nse2d_plan* best, double* ms_per_step, cudaStream_t s);
/* As nse2d_step without a graph, and the last step also stores its stage-3 rhs in the
 * context (field 4), which the next nse2d_diagnostics(t0_row = 0) pairs with omega for the
 * dOmega_rhs column (src/main.cu:586). */
int  nse2d_step_store_rhs(nse2d_ctx* ctx, int nsteps, cudaStream_t s);
/* As nse2d_step without a graph, with CUDA events on s around every kernel; kernel_ms[k]
 * receives the summed duration of the k-th kernel of a step over the nsteps steps
 * (nse2d_launches_per_step entries). Synchronous. */
int  nse2d_step_timed(nse2d_ctx* ctx, int nsteps, double* kernel_ms, cudaStream_t s);
/* One step (storing its stage-3 rhs, as nse2d_step_store_rhs) with CUDA events around every
 * kernel: the step's device time, the time of its row transforms and of its tridiagonal
 * solves, in ms (the step_ms, fft_ms and tridiag_ms columns of the reference's timing.csv,
 * src/main.cu:746-753; any output may be NULL). Synchronous. */
int  nse2d_step_profiled(nse2d_ctx* ctx, double* step_ms, double* fft_ms, double* tridiag_ms,
                         cudaStream_t s);
/* Name of the k-th kernel of a step. */
const char* nse2d_step_kernel_name(nse2d_ctx* ctx, int k);
/* Number of kernels one step launches. */
int  nse2d_launches_per_step(nse2d_ctx* ctx);
int  nse2d_set_dt(nse2d_ctx* ctx, double dt, cudaStream_t s);
/* Output times used for dt trimming and the snap after a step (1e300 = none). */
int  nse2d_set_schedule(nse2d_ctx* ctx, double next_snap, double next_diag, cudaStream_t s);
/* Read t, dt, step count and the last max |u|, |v|, |v| a (any may be NULL). Synchronous. */
int  nse2d_get_time(nse2d_ctx* ctx, double* t, double* dt, long long* step, double* umax3,
                    cudaStream_t s);

/* Run the time loop on the device (src/main.cu:434-551) until something needs the host:
 * steps are taken inside one CUDA graph launch (a WHILE node around the captured step) and
 * the run stops after the step at which
 *   NSE2D_HALT_OUTPUT     t has reached min(next_snap, next_diag) (within the snap tolerance),
 *   NSE2D_HALT_STATS      the step count is a multiple of stats_every (0: never),
 *   NSE2D_HALT_END        t >= t_end - dt/2 (the reference's loop test),
 *   NSE2D_HALT_NONFINITE  a bounded wait timed out, or the max reduction of an adaptive step saw
 *                         NaN/Inf in psi for the first time since the state was set (a run halts
 *                         once for that; nse2d_nonfinite tells the two apart),
 *   NSE2D_HALT_BUDGET     max_steps steps were taken;
 * *reason receives those bits. dt is trimmed to the output times as in the reference. At least
 * one step is taken. Synchronous. */
#define NSE2D_HALT_OUTPUT    1
#define NSE2D_HALT_STATS     2
#define NSE2D_HALT_END       4
#define NSE2D_HALT_NONFINITE 8
#define NSE2D_HALT_BUDGET    16
int  nse2d_run(nse2d_ctx* ctx, double next_snap, double next_diag, int stats_every, double t_end,
               long long max_steps, int* reason, cudaStream_t s);
/* Row sums over x of u, v, u^2, v^2 and u v of the current psi (src/diag.cu:468-499), neighbours
 * clamped at the walls: out5 = [5][Ny] host array. Synchronous. */
int  nse2d_row_moments(nse2d_ctx* ctx, double* out5, cudaStream_t s);
/* The time-weighted statistics of the reference's loop (src/main.cu:695-733) kept on the device:
 * with every > 0, every `every` steps of nse2d_run (the step count a multiple of every) the row
 * means over x of u, v, u^2, v^2, u v of that step's psi, weighted by the time since the last
 * sample, are added to an accumulator inside the run's graph, so that statistics need no halt of
 * the run (its stats_every argument may then be 0). The accumulator starts at zero and the clock
 * at the current t with this call; every = 0 turns it off. Setting a new state (nse2d_set_omega /
 * nse2d_set_state) turns it off. Precision 64 only. Synchronous. */
int  nse2d_stats_device(nse2d_ctx* ctx, int every, cudaStream_t s);
/* The accumulated statistics: out5 = [5][Ny] (the sums H[q][j] of the reference's loop; either
 * output may be NULL) and the total weight T (profiles = H / T). Synchronous. */
int  nse2d_stats_read(nse2d_ctx* ctx, double* out5, double* T, cudaStream_t s);
/* Add one sample of the 1-D spectra E_u(k), E_v(k) of the current psi (src/diag.cuh:123-191,
 * src/diag.cu:868-898), with the project's own row FFT. Overwrites the stage buffers (fields 2
 * and 3); call between steps. */
int  nse2d_spectra_accumulate(nse2d_ctx* ctx, cudaStream_t s);
/* kx = 2 pi k / Lx and the sample-averaged spectra, k = 0..Nx/2 (Nx/2+1 values each; any
 * output may be NULL); *samples receives the sample count. Synchronous. */
int  nse2d_spectra(nse2d_ctx* ctx, double* kx, double* Eu, double* Ev, int* samples, cudaStream_t s);

/* Poisson solve of the reference (src/poisson.cuh:83-118): psi from omega, Dirichlet
 * psi = 0 / 2 h Ub at the walls on kx = 0. Device pointers, asynchronous. */
int  nse2d_poisson_solve(nse2d_ctx* ctx, const double* d_w, double* d_psi, cudaStream_t s);
/* max |u|, |v|, |v| a of the context's psi (src/diag.cu:821-866). Synchronous. */
int  nse2d_max_uv(nse2d_ctx* ctx, double* out3, cudaStream_t s);
/* The same max |u|, |v|, |v| a of a caller-owned psi [Ny][Nx] and a_node [Ny] (device
 * pointers), without a context and without allocating any device memory. No counterpart in
 * the reference. It is for callers that may not allocate: code whose device memory is all
 * handed out by its own pool, or that cannot afford the device-wide synchronisation of a
 * cudaMalloc/cudaFree pair in its loop. The reduction's scratch is a small control block
 * inside the library (the CTAs combine their maxima there by atomic max); the launch uses at
 * most NSE2D_MAXUV_NOALLOC_MAX_BLOCKS CTAs, which stride over the rows, so every grid fits.
 * Nx must be in [2, 2^30] and Ny >= 3, and both pointers 8-byte aligned (any Nx and offset
 * work; 16-byte loads are used where Nx is even and psi 16-byte aligned); other arguments are
 * rejected with an error (status -1).
 * The first call on a device (with that device current) looks up the scratch address; it is
 * also where CUDA, which loads a library's kernels on first use, places this entry point's
 * code and the static scratch on that device (a one-time placement by the driver): callers
 * that must see no change of free device memory later make one call during their set-up.
 * Every call clears the control block on stream s first. One scratch serves all callers on a
 * device: calls that overlap in time on the same device race. Synchronous (it ends with a copy
 * to host memory and a stream synchronisation): it must not be called while any stream of the
 * device is being captured. Returns 0, or NSE2D_STATUS_NONFINITE when psi holds NaN or Inf
 * (out3 then holds the maxima of the finite differences). */
#define NSE2D_MAXUV_NOALLOC_MAX_BLOCKS 1024
#define NSE2D_STATUS_NONFINITE 2
int  nse2d_max_uv_noalloc(const double* d_psi, const double* d_a_node, int Nx, int Ny,
                          double inv_dx, double inv_deta, double* out3, cudaStream_t s);
/* One diagnostics.csv row at the current state, columns umax .. Re_tau (16) followed by
 * the 13 closure_diag columns (nan when not computed), as src/main.cu:566-692
 * (t0_row = 0) or the t = 0 row of src/main.cu:325-421 (t0_row = 1). Synchronous. */
int  nse2d_diagnostics(nse2d_ctx* ctx, int t0_row, double* out29, cudaStream_t s);
/* J and rhs at the context's state and time t into fields 5 and 4. Synchronous. */
int  nse2d_rhs_at_state(nse2d_ctx* ctx, double t, cudaStream_t s);
/* u, v of the context's psi into caller device arrays (src/ops.cu:47-70). */
int  nse2d_uv(nse2d_ctx* ctx, double* d_u, double* d_v, cudaStream_t s);
/* Non-finite and timeout flags since the state was last set (nse2d_set_omega / nse2d_set_state):
 * bit 0 a max reduction met NaN or Inf in psi, bit 1 a bounded wait of a kernel timed out.
 * Synchronous. */
int  nse2d_nonfinite(nse2d_ctx* ctx, int* flag, cudaStream_t s);
/* Host copy of a metric: 0 y, 1 a_node, 2 a_edge (Ny-1), 3 dy_edge (Ny-1), 4 w_node. */
int  nse2d_metrics(nse2d_ctx* ctx, int which, double* out);
/* Scalars: 0 nu, 1 dx, 2 deta, 3 invA_full, 4 meanFx_A, 5 psi_bot, 6 psi_top. */
int  nse2d_scalar(nse2d_ctx* ctx, int which, double* out);

/* ---------------------------------------------------------------------------------------
 * 3. Batched ensembles (no counterpart in the reference, which runs one channel per process)
 * ------------------------------------------------------------------------------------- */
/* Many independent channels advanced by one graph launch: members are existing contexts (each
 * with its own grid, physics, state and adaptive dt), which must outlive the ensemble. The
 * graph's WHILE node repeats one step of every member; members are dealt round-robin onto
 * `groups` concurrent branches. Results do not depend on the grouping. Creating the ensemble
 * sets its members to the two-pass tridiagonal solve (nse2d_set_tridiag_form(m, 0)), whose
 * plain grids share the device with the other branches. */
typedef struct nse2d_ensemble nse2d_ensemble;
int  nse2d_ensemble_create(nse2d_ctx* const* members, int n, nse2d_ensemble** out);
int  nse2d_ensemble_destroy(nse2d_ensemble* e);
/* Advance every member by nsteps steps in one graph launch, asynchronously on s. */
int  nse2d_ensemble_step(nse2d_ensemble* e, int nsteps, cudaStream_t s);
/* Use `groups` concurrent branches (1..n; rebuilds the graph). */
int  nse2d_ensemble_set_groups(nse2d_ensemble* e, int groups);
/* Time every power-of-two branch count (and n) over trial_steps steps each, keep the fastest,
 * and report it and its time per ensemble step. The trials are real steps of every member
 * (1 + trial_steps per candidate). Synchronous. */
int  nse2d_ensemble_autotune(nse2d_ensemble* e, int trial_steps, int* groups_out, double* ms_per_step_out,
                             cudaStream_t s);
/* The branch count as nse2d_ensemble_autotune, then the kernel plans of the members (nse2d_plan):
 * for each class of members with the same grid and precision, every form the class can switch is
 * toggled for the whole class and kept if the timed ensemble step is faster (coordinate
 * descent), then the branch count is tuned again. The trials are real steps of every member.
 * nse2d_get_plan reports each member's chosen plan. Synchronous. */
int  nse2d_ensemble_autotune_plans(nse2d_ensemble* e, int trial_steps, int* groups_out, double* ms_per_step_out,
                                   cudaStream_t s);

/* ---- 4. Learned subgrid closure (no reference counterpart) ----
 * BF16 operands on the 5th-generation tensor cores (tcgen05), FP32 accumulate. */

/* C[M][ldc] = A[M][K] . B[N][K]^T (+ bias[N]), all device pointers, A and B BF16 row-major
 * (K contiguous, 16-byte aligned). Cf (FP32, before the activation) and Cb (BF16, after it:
 * ReLU when relu != 0) may each be NULL. M a multiple of 128, N a multiple of 16 in [16, 256],
 * K a multiple of 64 (pad with zeros). Synchronous: returns nonzero if a bounded wait ran out. */
int  nse2d_gemm_bf16(const void* A, const void* B, const float* bias, float* Cf, void* Cb, int M, int N, int K,
                     int ldc, int relu, cudaStream_t s);

/* Top-hat filter of a fine field [Nyf][Nxf] onto the coarse grid whose nodes are every
 * Nxf/Nxc-th column and (Nyf-1)/(Nyc-1)-th row (device pointers): the mean over the fine
 * points within half a coarse cell, half weight on the cell edges, periodic in x, rows beyond
 * the walls left out. */
int  nse2d_box_filter(const double* fine, int Nxf, int Nyf, double* coarse, int Nxc, int Nyc, cudaStream_t s);

/* The closure model on an Nx x Ny coarse grid: four 3x3 convolutions 5 -> hidden -> hidden ->
 * hidden -> 1 (GELU, tanh form, after the first three; x periodic, zero beyond the walls) from
 * (omega / s0, psi / s1, u / s2, v / s3, y) to tau / tau_scale, where tau = filter(J(psi, omega))
 * - J(filter psi, filter omega) is the subgrid part of the Jacobian. Convolutions are BF16
 * GEMMs on the tensor cores with FP32 accumulate; weights are kept in FP32 and trained with
 * AdamW on batches of up to max_batch whole fields. hidden is a multiple of 16 in [16, 64]; y
 * is the host array of the Ny wall-normal coordinates. Weights are passed as [cout][9][cin]
 * (tap = 3 (dy + 1) + dx + 1) and biases as [cout], on the host. Field pointers are device
 * pointers, FP64: one field [Ny][Nx], or S samples [S][Ny][Nx] with the batch's sample
 * indices idx[nb] (host). */
typedef struct nse2d_cnn nse2d_cnn;
int  nse2d_cnn_create(int Nx, int Ny, int hidden, int max_batch, const double* y, nse2d_cnn** out);
int  nse2d_cnn_destroy(nse2d_cnn* c);
int  nse2d_cnn_layer_shape(nse2d_cnn* c, int layer, int* cin, int* cout);
int  nse2d_cnn_set_params(nse2d_cnn* c, int layer, const float* w, const float* b);
int  nse2d_cnn_get_params(nse2d_cnn* c, int layer, float* w, float* b);
/* gradients of the last nse2d_cnn_gradients / nse2d_cnn_train_step */
int  nse2d_cnn_get_grads(nse2d_cnn* c, int layer, float* w, float* b);
/* in_scales: the 4 scales of omega, psi, u, v */
int  nse2d_cnn_set_scales(nse2d_cnn* c, const double* in_scales, double tau_scale);
/* Where the model acts: tau = 0 on the wall_rows rows next to each wall (the wall row
 * included; default 1), in the loss and in the output; the output is multiplied by gain
 * (default 1); with row_mean != 0 every row of the output is replaced by its x-mean (the
 * mean-flow part of tau, which is what the mean velocity and Re_tau see). */
int  nse2d_cnn_set_application(nse2d_cnn* c, int wall_rows, double gain, int row_mean);
/* tau (FP64, zero on the wall rows) from one field's omega, psi, u, v; asynchronous and
 * graph-capturable */
int  nse2d_cnn_forward(nse2d_cnn* c, const double* w, const double* psi, const double* u, const double* v, double* tau,
                       cudaStream_t s);
/* loss = mean over the interior pixels of the batch of (output - tau / tau_scale)^2 and its
 * gradients; waits, and stores the loss when loss != NULL */
int  nse2d_cnn_gradients(nse2d_cnn* c, const double* w, const double* psi, const double* u, const double* v,
                         const double* tau, const int* idx, int nb, float* loss, cudaStream_t s);
/* gradients, then one AdamW step (beta1 0.9, beta2 0.999, eps 1e-8, decoupled weight decay) */
int  nse2d_cnn_train_step(nse2d_cnn* c, const double* w, const double* psi, const double* u, const double* v,
                          const double* tau, const int* idx, int nb, float lr, float weight_decay, float* loss,
                          cudaStream_t s);
/* Attach a model of the context's grid (NULL detaches): tau is subtracted from the rhs of the
 * interior rows. every_stage != 0: the model runs before every stage on that stage's psi,
 * omega^(s); 0: it runs once per step on psi^n, omega^n and its tau is held over the three
 * stages. Precision 64. */
int  nse2d_set_closure(nse2d_ctx* ctx, nse2d_cnn* net, int every_stage);

/* ---- 5. Snapshot files (host code; no GPU) ----
 * The reference's HDF5 snapshot layout (src/io.cu:183-259): datasets omega, psi, u, v
 * [Ny][Nx] float64 (any subset, omega first), y [1][Ny] with attributes beta and stretch_code
 * when stretch_tanh and y are given, root attributes t, Nx, Ny (int32), Lx, Ly, h, dx, dy, nu;
 * written without libhdf5 (superblock 0, symbol-table root group, contiguous datasets), read as
 * the reference reads it (src/init.cu:215-279). format 1 is the flat "bin" layout of the
 * reference's declared SNAP_BIN (src/io.cuh:28), which it never writes. */
typedef struct nse2d_snapshot_meta {
    int    Nx, Ny;
    double t, Lx, h, nu, beta;
    int    stretch_tanh;      /* 1: tanh grid (y and its attributes are written when y != NULL) */
    const double* y;          /* write: the Ny node coordinates, or NULL; read: set to NULL */
    int    fields;            /* read: bits 1 omega, 2 psi, 4 u, 8 v, 16 y present */
} nse2d_snapshot_meta;
/* format 0: HDF5, 1: bin. At most 8 fields of Ny x Nx values each. */
int  nse2d_snapshot_write(const char* path, int format, const nse2d_snapshot_meta* m, int nfields,
                          const char* const* names, const double* const* fields);
/* Either format (told apart by the file's signature). m (may be NULL) receives the metadata;
 * with name != NULL the field ("omega", "psi", "u", "v": Ny x Nx values, stored [Ny][Nx] or
 * transposed; "y": Ny values) is copied to out. */
int  nse2d_snapshot_read(const char* path, nse2d_snapshot_meta* m, const char* name, double* out);

const char* nse2d_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* NSE2D_B200_H */
