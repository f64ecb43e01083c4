// Common types of the B200 channel time step: the solver context, its device control
// block and error handling. Written for this project.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include <cuda.h>

#include "fft.cuh"

namespace nse2d {

// ---- error handling: every entry point returns a status; the message is kept per thread ----
void set_error(const char* fmt, ...);
const char* get_error();

#define NSE_CUDA_TRY(expr)                                                                       \
    do {                                                                                         \
        cudaError_t e__ = (expr);                                                                \
        if (e__ != cudaSuccess) {                                                                \
            ::nse2d::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e__)); \
            return -1;                                                                           \
        }                                                                                        \
    } while (0)

// ---- run configuration (the reference's Grid + Params, src/common.cuh:42-114) ----
struct Config {
    int Nx = 1024, Ny = 1025;
    double Lx = 12.566370612, h = 1.0;
    int stretch = 0;         // 0 none, 1 tanh
    double beta = 0.0;
    double Ub = 1.0, Reb = 10000.0, nu_override = -1.0;
    double dt_init = 1e-3, dt_max = 1e-2, cfl = 0.5, cvisc = 0.5;
    int adapt = 1;
    double t_end = 200.0, F0 = 0.0;
    int nforce = 1;
    double lin_drag = 0.0;
    int free_slip = 0, mms = 0;
    double mms_A0 = 1e-3, mms_eps = 0.1, mms_Om = 1.0;
    int mms_kx = 1, closure_diag = 0;
    int precision = 64;      // 64: FP64 throughout; 32: FP32 bulk with FP64 islands
    std::vector<double> y_table;   // stretch 2: the Ny node coordinates
    // metrics given by the caller (Poisson2D_Z2Z::enable_mapped): a_node [Ny] and a_edge [Ny-1]
    // replace the built ones (y and the weights stay those of the stretch)
    std::vector<double> a_node_in, a_edge_in;
};

// Device control block: time, step size and the step's reductions. Kept on the device so
// that a sequence of steps (with adaptive dt) needs no host round trip and can be captured
// in a CUDA graph.
struct Ctl {
    double t, dt;
    double umax, vmax, vmaxm;      // max |u|, |v|, |v| a of the last reduction
    double next_out;               // next output time for dt trimming (1e300: none)
    double next_snap, next_diag;   // scheduled output times for the snap after a step (1e300: none)
    double jwall[3];               // closure_diag: enstrophy added by the wall update, per stage
    long long step;
    unsigned int blocks_done;      // last-block-done counter of the max reduction
    unsigned int ifft_done;        // last-block-done counter of the stage-3 inverse transform
    unsigned int thom_done[2];     // inverse transform: rows 1-2 / Ny-3..Ny-2 written (per wall)
    unsigned long long mx_acc[3];  // max reduction: atomic maxima of |u|, |v|, |v| a (bit patterns; 0 between launches)
    int nonfinite;                 // bit 0: a reduction saw NaN/Inf; bit 1: a bounded wait timed out
    int nonfinite_halted;          // a run has already halted for bit 0 (it halts once for it)
    // statistics on the device (nse2d_stats_device): every acc_every steps of a run, the row
    // moments weighted by t - acc_last_t are added to the context's accumulator
    int acc_every;
    double acc_last_t, acc_T;
    double mx_next[3];             // max |u|, |v|, |v| a of the current psi (the next step's dt)
    // run mode (nse2d_run): stop stepping when an output, a statistics step or the end is due
    int run;                       // 1 while a run is active
    int halt;                      // set at the end of the step after which the run stops
    int halt_reason;               // NSE2D_HALT_* bits
    int stats_every;               // steps between statistics samples (0: none)
    long long run_budget;          // steps a run may still take (a hard bound on the device loop)
    double t_end;                  // the loop runs while t < t_end - dt/2 (src/main.cu:434)
};

// Row-constant tables (device), length Ny unless noted.
struct RowTables {
    double* y;          // node coordinates
    double* a_node;     // eta_y at nodes
    double* a_edge;     // eta_y at j+1/2 (Ny-1)
    double* dy_edge;    // y_{j+1}-y_j (Ny-1)
    double* w_node;     // trapezoid weights
    double* wt_node;    // deta / a_node on interior rows, 0 at walls
    double* frow;       // vorticity forcing f(y_j)
    double* st_cj;      // stage stencil: a_j inv_dx inv_deta / 12 (the Arakawa factor a / (4 dx deta) / 3)
    double* st_ap;      // stage stencil: nu a_j a_{j+1/2} / deta^2
    double* st_am;      // stage stencil: nu a_j a_{j-1/2} / deta^2
    double* asub;       // Thomas sub-diagonal a_j a_{j-1/2} / deta^2
    double* csup;       // Thomas super-diagonal a_j a_{j+1/2} / deta^2
    double* inv_csup;   // 1 / csup
    // MMS tables (only when mms): per row g, g'', sin(2 theta); per column sin(kx), sin(2kx)
    double* mms_g;
    double* mms_gpp;
    double* mms_sin2;
    double* mms_sk;
    double* mms_s2k;
};

struct Context {
    Config cfg;
    int Nx = 0, Ny = 0, M = 0, H = 0, Hp = 0, Ni = 0;
    size_t N = 0;
    double dx = 0, dy = 0, inv_dx = 0, inv_dx2 = 0, deta = 0, inv_deta = 0, inv_deta2 = 0;
    double nu = 0, dy_min = 0, inv_dymin2 = 0, Ly_full = 0, invA_full = 0, meanFx_A = 0;
    double psi_bot = 0, psi_top = 0;
    // host copies of the metrics
    std::vector<double> h_y, h_a_node, h_a_edge, h_dy_edge, h_w_node;
    RowTables rt{};
    // fields (FP64 state), owned by the context
    double *w = nullptr, *w1 = nullptr, *w2 = nullptr, *psi = nullptr;
    // scratch used by diagnostics: rhs and J at one state, and the stage-3 rhs of the last step
    double *rhs = nullptr, *J = nullptr;
    // spectral buffer [Ny][Hp] complex, FP64 (in place: omega-hat in, psi-hat out)
    cpx<double>* hat = nullptr;
    double* cp = nullptr;          // elimination table [Ni][Hp]
    cpx<double>* tw = nullptr;     // per-pass twiddle pairs of the Nx/2-point transform
    cpx<double>* wN = nullptr;     // M+1 twiddles e^{-2 pi i k/Nx}
    // reductions
    double* red_blocks = nullptr;  // per-block partials (max and diagnostics)
    double* red_out = nullptr;     // reduced values
    int red_nblocks = 0;
    size_t red_capacity = 0;       // doubles in red_blocks
    Ctl* ctl = nullptr;            // device control block
    Ctl* h_ctl = nullptr;          // pinned host mirror
    // launch shapes
    int fft_threads = 256;
    int stage_grid = 0, ifft_grid = 0;
    // segmented Thomas solve: 16-column groups, segments of TS_ROWS rows, blocks of TS_NW segments (one CTA)
    int thomas_groups = 0, thomas_nseg = 0, thomas_nsb = 0;
    double* tconst = nullptr;      // [nseg][3][Hp] segment products P, V, Q
    double* tmaps = nullptr;       // [nseg][2][2 Hp] segment maps D, U
    double* tblk = nullptr;        // [groups][nsb][5][32] block aggregates
    double* tbcarry = nullptr;     // [groups][nsb][2][32] block carries c, X
    unsigned int* tcount = nullptr;  // [groups] arrival counters (zero between solves)
    // one-pass cluster solve (k_thomas_cluster<L>): CTAs per cluster, rows per segment, resident
    // clusters (the persistent grid), dynamic shared memory, TMA maps of omega-hat and cp
    bool thomas_cluster = false;   // the form the step uses (nse2d_set_tridiag_form)
    bool thomas_cluster_ok = false;  // the cluster form can be resident on this device
    int tc_cluster = 0, tc_L = 0, tc_nclusters = 0;
    size_t tc_smem = 0;
    CUtensorMap tm_hat{}, tm_cp{};
    // precision 32: the FP32 spectral buffer [Ny][Hp] and the cluster solve's map and sizes for it
    cpx<float>* hat32 = nullptr;
    CUtensorMap tm_hat32{};
    size_t tc_smem32 = 0;
    int tc_nclusters32 = 0;
    int num_sms = 0;
    int maxuv_ctas = 0;            // resident CTAs of k_maxuv_dt (occupancy x SMs)
    // learned closure: the model evaluated before every stage and its output tau [Ny][Nx]
    struct Cnn* closure_net = nullptr;
    double* closure_tau = nullptr;       // tau, then the u, v scratch of the model's inputs
    bool closure_every_stage = true;     // false: tau of the step's first stage for all three
    // FP32-bulk variant (precision 32): base profiles (FP64) and FP32 fluctuations
    bool prec32 = false;
    float *wf = nullptr, *w1f = nullptr, *w2f = nullptr, *psif = nullptr, *rhsf = nullptr;
    double *wbar = nullptr, *psibar = nullptr;
    float* rc32 = nullptr;                 // [RC32_N][Ny] row constants of the FP32 stage
    cpx<float> *twf = nullptr, *wNf = nullptr;
    double wall_bot32 = 0.0, wall_top32 = 0.0;
    int maxuv32_ctas = 0;          // resident CTAs of k_maxuv32 (occupancy x SMs)
    // FP32 stage kernel: TMA tensor maps of psi' and of the three w' buffers (Nx >= 256)
    bool stage32_tma = false, stage32_tma_ok = false;
    int stage32_tma_grid = 0;
    CUtensorMap tm32_psi{}, tm32_w[3]{}, tm32_wn{};
    // row transforms at Nx = 4096: the forms whose rows are prefetched by bulk copies
    bool rowfft_pf = false, rowfft_pf_ok = false;
    bool max_fused = false;          // with rowfft_pf, adaptive FP64: max reduction in the stage-3 inverse transform
                                     // (off by default: measured slower than the separate reduction at 4096x2049)
    bool pdl = false;                // step kernels launched with programmatic dependent launch
    unsigned int* bcount = nullptr;  // [grid + 1] band-boundary counters of the fused max reduction
    // stage kernel: TMA tensor maps of psi and of the three omega buffers (Nx >= 128)
    bool stage_tma = false, stage_tma_ok = false;
    int stage_tma_grid = 0;
    CUtensorMap tm_psi{}, tm_w[3]{}, tm_wn{};
    cudaStream_t cap_stream = nullptr;     // private stream used only for graph capture
    cudaGraphExec_t graph_exec = nullptr;  // one captured step
    cudaGraphExec_t run_exec = nullptr;    // WHILE(no halt) { step } for nse2d_run
    double* spec_acc = nullptr;            // [2][Hp] accumulated E_u, E_v of the 1-D spectra
    double* moments = nullptr;             // [5][Ny] row sums of u, v, u^2, v^2, u v
    double* stats_acc = nullptr;           // [5][Ny] time-weighted row means (statistics on the device)
    bool stats_dev = false;                // the run graph accumulates the statistics
    int spec_samples = 0;
    bool closure_diag = false;
};

}  // namespace nse2d
