// Solver context: grid metrics, tables, device buffers and the enqueueing of one
// SSPRK(3,3) step. Written for this project; the setup follows the reference's
// src/grid.cu:7-94 (metrics), src/main.cu:49-87 (derived constants), src/poisson.cu:16-68
// (kx^2 and the elimination table) and src/main.cu:210-213 (initial solve + Thom).
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>

#include <cudaTypedefs.h>

#include "nse2d_internal.h"
#include "step_kernels.cuh"

namespace nse2d {

static thread_local char g_err[1024] = "";
void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char* get_error() { return g_err; }

// ---- grid metrics on the host: src/grid.cu:7-94 ----
int build_y_metrics(const Config& c, std::vector<double>& y, std::vector<double>& a_node,
                    std::vector<double>& a_edge, std::vector<double>& dy_edge, std::vector<double>& w_node) {
    const int Ny = c.Ny;
    const double h = c.h;
    y.assign(Ny, 0.0); a_node.assign(Ny, 0.0); a_edge.assign(Ny - 1, 0.0);
    dy_edge.assign(Ny - 1, 0.0); w_node.assign(Ny, 0.0);
    if (Ny <= 2 || c.stretch == 0) {
        const double dy = (2.0 * h) / (double)(Ny - 1);
        for (int j = 0; j < Ny; ++j) y[j] = -h + j * dy;
        const double deta = 2.0 / (double)(Ny - 1);
        const double y_eta = dy / deta;
        const double a = 1.0 / y_eta;
        for (int j = 0; j < Ny; ++j) a_node[j] = a;
        for (int j = 0; j < Ny - 1; ++j) { a_edge[j] = a; dy_edge[j] = dy; }
        for (int j = 0; j < Ny; ++j) w_node[j] = dy;
        w_node[0] *= 0.5; w_node[Ny - 1] *= 0.5;
        return 0;
    }
    if (c.stretch == 2) {
        // tabulated y (src/grid.cu:46-78): a = 1 / y_eta with y_eta by differences in eta,
        // one-sided at the walls, central inside
        if ((int)c.y_table.size() != Ny) {
            set_error("stretch 2 (table) needs y_table with Ny = %d values", Ny);
            return -1;
        }
        y = c.y_table;
        const double deta = 2.0 / (double)(Ny - 1);
        for (int j = 0; j < Ny; ++j) {
            double yeta;
            if (j == 0) yeta = (y[1] - y[0]) / deta;
            else if (j == Ny - 1) yeta = (y[Ny - 1] - y[Ny - 2]) / deta;
            else yeta = (y[j + 1] - y[j - 1]) / (2.0 * deta);
            a_node[j] = 1.0 / yeta;
        }
    } else if (c.stretch != 1) {
        set_error("unknown stretch code %d (0 none, 1 tanh, 2 table)", c.stretch);
        return -1;
    } else {
        const double b = (c.beta > 0 ? c.beta : 2.5);
        for (int j = 0; j < Ny; ++j) {
            const double e = -1.0 + 2.0 * (double)j / (double)(Ny - 1);
            y[j] = h * std::tanh(b * e) / std::tanh(b);
        }
        for (int j = 0; j < Ny; ++j) {
            const double e = -1.0 + 2.0 * (double)j / (double)(Ny - 1);
            const double sech = 1.0 / std::cosh(b * e);
            a_node[j] = 1.0 / (h * b * (sech * sech) / std::tanh(b));
        }
    }
    for (int j = 0; j < Ny - 1; ++j) a_edge[j] = 0.5 * (a_node[j] + a_node[j + 1]);
    for (int j = 0; j < Ny - 1; ++j) dy_edge[j] = y[j + 1] - y[j];
    w_node[0] = 0.5 * dy_edge[0];
    w_node[Ny - 1] = 0.5 * dy_edge[Ny - 2];
    for (int j = 1; j < Ny - 1; ++j) w_node[j] = 0.5 * (dy_edge[j - 1] + dy_edge[j]);
    return 0;
}

// the metrics of a context: those of the stretch, or the caller's a_node / a_edge where given
static int context_metrics(const Config& c, std::vector<double>& y, std::vector<double>& a_node,
                           std::vector<double>& a_edge, std::vector<double>& dy_edge, std::vector<double>& w_node) {
    if (build_y_metrics(c, y, a_node, a_edge, dy_edge, w_node)) return -1;
    if (!c.a_node_in.empty()) {
        if ((int)c.a_node_in.size() != c.Ny || (int)c.a_edge_in.size() != c.Ny - 1) {
            set_error("given metrics must have Ny and Ny-1 values");
            return -1;
        }
        a_node = c.a_node_in;
        a_edge = c.a_edge_in;
    }
    return 0;
}

using ThomasClusterKernel = void (*)(ThomasMaps, ThomasParams);
template <bool F32> static ThomasClusterKernel thomas_cluster_kernel_t(int L) {
    switch (L) {
        case 1: return k_thomas_cluster<1, F32>;
        case 2: return k_thomas_cluster<2, F32>;
        case 4: return k_thomas_cluster<4, F32>;
        case 8: return k_thomas_cluster<8, F32>;
        case 16: return k_thomas_cluster<16, F32>;
        default: return nullptr;
    }
}
static ThomasClusterKernel thomas_cluster_kernel(int L, bool f32 = false) {
    return f32 ? thomas_cluster_kernel_t<true>(L) : thomas_cluster_kernel_t<false>(L);
}

// homog: the FP32-bulk step's solve, for psi' (zero on the walls) in the FP32 spectral buffer
static ThomasParams thomas_params(const Context* c, bool homog = false) {
    ThomasParams p{};
    p.hat = c->hat; p.hat32 = c->hat32; p.cp = c->cp; p.asub = c->rt.asub; p.inv_csup = c->rt.inv_csup; p.csup = c->rt.csup;
    p.tconst = c->tconst; p.tmaps = c->tmaps; p.tblk = c->tblk; p.tbcarry = c->tbcarry; p.tcount = c->tcount;
    p.Nx = c->Nx; p.Ny = c->Ny; p.Hp = c->Hp; p.H = c->H; p.Ni = c->Ni;
    p.nseg = c->thomas_nseg; p.nsb = c->thomas_nsb;
    p.ctl = c->ctl;
    p.psi_bot = homog ? 0.0 : c->psi_bot;
    p.psi_top = homog ? 0.0 : c->psi_top;
    return p;
}

// ---- device setup kernels ----
// Elimination table, one thread per kx: src/poisson.cu:16-22 (kx^2) and :38-68 (cp), the
// same expressions; stored [Ni][Hp] so that a warp reads consecutive kx.
__global__ void k_setup_cp(double* cp, const double* a_node, const double* a_edge, int Nx, int Ny,
                           int Hp, int H, double Lx, double inv_deta2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= H) return;
    const int Ni = Ny - 2;
    const int kphys_i = (k <= Nx / 2 ? k : k - Nx);
    const double kphys = (2.0 * kPiD * (double)kphys_i) / Lx;
    const double kx2 = kphys * kphys;
    int j = 1;
    double an = a_node[j], ae_p = a_edge[j], ae_m = a_edge[j - 1];
    double a_sub = an * ae_m * inv_deta2, c_sup = an * ae_p * inv_deta2;
    double b = -(a_sub + c_sup) - kx2;
    double cp_prev = c_sup / b;
    cp[k] = cp_prev;
    for (int r = 1; r < Ni; ++r) {
        j = r + 1;
        an = a_node[j]; ae_p = a_edge[j]; ae_m = a_edge[j - 1];
        a_sub = an * ae_m * inv_deta2; c_sup = an * ae_p * inv_deta2;
        b = -(a_sub + c_sup) - kx2;
        const double den = b - a_sub * cp_prev;
        const double cpi = c_sup / den;
        cp[(size_t)r * Hp + k] = cpi;
        cp_prev = cpi;
    }
}

// Row tables: Thomas coefficients (poisson.cu:86-88), forcing f(y) (ops.cu:526-531), trapezoid
// weights wt (main.cu:252-254) and the MMS row factors (ops.cu:587-603).
__global__ void k_setup_rows(RowTables rt, int Ny, double inv_deta2, double deta, double F0, int nforce,
                             double h, double mms_k, double mms_c, double inv4dxde, double nu) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Ny) return;
    if (j >= 1 && j <= Ny - 2) {
        const double an = rt.a_node[j];
        rt.asub[j] = an * rt.a_edge[j - 1] * inv_deta2;
        rt.csup[j] = an * rt.a_edge[j] * inv_deta2;
        rt.inv_csup[j] = 1.0 / rt.csup[j];
        rt.wt_node[j] = deta / an;
        rt.st_cj[j] = an * (inv4dxde * (1.0 / 3.0));
        rt.st_ap[j] = nu * (an * rt.a_edge[j] * inv_deta2);
        rt.st_am[j] = nu * (an * rt.a_edge[j - 1] * inv_deta2);
    } else {
        rt.asub[j] = 0.0; rt.csup[j] = 0.0; rt.inv_csup[j] = 0.0; rt.wt_node[j] = 0.0;
        rt.st_cj[j] = 0.0; rt.st_ap[j] = 0.0; rt.st_am[j] = 0.0;
    }
    double f = 0.0;
    if (F0 != 0.0) {
        const double yy = rt.y[j];
        const double arg = (double)nforce * kPiD * ((yy + h) / (2.0 * h));
        f = -F0 * ((double)nforce * kPiD / (2.0 * h)) * cos(arg);
    }
    rt.frow[j] = f;
    if (rt.mms_g) {
        const double theta = mms_c * (rt.y[j] + h);
        const double two_th = 2.0 * theta;
        const double s_th = sin(theta);
        const double s = s_th * s_th;
        const double cos2 = cos(two_th), sin2 = sin(two_th);
        const double c2 = mms_c * mms_c;
        rt.mms_g[j] = (mms_k * mms_k) * s - 2.0 * c2 * cos2;
        rt.mms_gpp[j] = 2.0 * c2 * cos2 * ((mms_k * mms_k) + 4.0 * c2);
        rt.mms_sin2[j] = sin2;
    }
}

__global__ void k_setup_mms_cols(double* sk, double* s2k, int Nx, double dx, double k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nx) return;
    const double x = (double)i * dx;
    sk[i] = sin(k * x);
    s2k[i] = sin(2.0 * k * x);
}

static void twiddles(int M, std::vector<cpx<double>>& tw, std::vector<cpx<double>>& wN) {
    const long double PI = 3.141592653589793238462643383279502884L;
    tw.resize(M);
    wN.resize(M + 1);
    for (int t = 0; t < M; ++t) {
        const long double a = -2.0L * PI * (long double)t / (long double)M;
        tw[t] = {(double)cosl(a), (double)sinl(a)};
    }
    for (int k = 0; k <= M; ++k) {
        const long double a = -PI * (long double)k / (long double)M;
        wN[k] = {(double)cosl(a), (double)sinl(a)};
    }
    tw[0] = {1.0, 0.0};
    if (M % 4 == 0) { tw[M / 4] = {0.0, -1.0}; tw[M / 2] = {-1.0, 0.0}; tw[3 * M / 4] = {0.0, 1.0}; }
    wN[0] = {1.0, 0.0};
    wN[M] = {-1.0, 0.0};
    if (M % 2 == 0) wN[M / 2] = {0.0, -1.0};
}

// 2-D tensor map of one [Ny][Nx] field (FP64, or FP32 with f32) with a box of bw x bh elements.
int encode_map_2d(CUtensorMap* map, const void* base, bool f32, int Nx, int Ny, int bw, int bh) {
    static PFN_cuTensorMapEncodeTiled encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            set_error("cuTensorMapEncodeTiled is not available from the driver");
            return -1;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)Nx, (cuuint64_t)Ny};
    const cuuint64_t strides[1] = {(cuuint64_t)Nx * (f32 ? sizeof(float) : sizeof(double))};
    const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                              const_cast<void*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (CUresult %d)", (int)r);
        return -1;
    }
    return 0;
}

static int encode_field_map(CUtensorMap* map, const double* base, int Nx, int Ny, int bw = SB_W, int bh = SB_H) {
    return encode_map_2d(map, base, false, Nx, Ny, bw, bh);
}

template <typename T> static int dalloc(T** p, size_t n) {
    NSE_CUDA_TRY(cudaMalloc((void**)p, n * sizeof(T) + 16));
    NSE_CUDA_TRY(cudaMemset(*p, 0, n * sizeof(T) + 16));
    return 0;
}

int context_create(const Config& cfg, Context** out) {
    *out = nullptr;
    if (cfg.Nx < 4 || (cfg.Nx & (cfg.Nx - 1)) != 0) {
        set_error("Nx = %d: the B200 path needs a power of two >= 4", cfg.Nx);
        return -1;
    }
    if (cfg.Ny < 5) { set_error("Ny = %d: need Ny >= 5", cfg.Ny); return -1; }
    if (cfg.Nx > 16384) { set_error("Nx = %d exceeds 16384", cfg.Nx); return -1; }
    if (cfg.precision != 64 && cfg.precision != 32) { set_error("precision %d: 64 or 32", cfg.precision); return -1; }
    if (cfg.precision == 32 && (cfg.mms || cfg.closure_diag)) {
        set_error("precision 32 (FP32 bulk) runs without the MMS forcing and the closure diagnostics");
        return -1;
    }
    auto* c = new Context();
    c->cfg = cfg;
    c->Nx = cfg.Nx; c->Ny = cfg.Ny; c->N = (size_t)cfg.Nx * cfg.Ny;
    c->M = cfg.Nx / 2; c->H = c->M + 1; c->Hp = (c->H + 15) / 16 * 16; c->Ni = cfg.Ny - 2;
    if (context_metrics(cfg, c->h_y, c->h_a_node, c->h_a_edge, c->h_dy_edge, c->h_w_node) != 0) { delete c; return -1; }
    const int Ny = c->Ny;
    c->nu = (cfg.nu_override >= 0 ? cfg.nu_override : (2.0 * cfg.h * cfg.Ub) / cfg.Reb);
    c->dx = cfg.Lx / (double)c->Nx;
    c->dy = (2.0 * cfg.h) / (double)(Ny - 1);
    c->inv_dx = 1.0 / c->dx; c->inv_dx2 = c->inv_dx * c->inv_dx;
    c->deta = 2.0 / (double)(Ny - 1);
    c->inv_deta = 1.0 / c->deta; c->inv_deta2 = c->inv_deta * c->inv_deta;
    c->dy_min = std::fabs(c->h_dy_edge[0]);
    for (int j = 1; j < Ny - 1; ++j) c->dy_min = std::min(c->dy_min, std::fabs(c->h_dy_edge[j]));
    c->inv_dymin2 = 1.0 / (c->dy_min * c->dy_min);
    c->Ly_full = 0.0;
    for (int j = 0; j < Ny; ++j) c->Ly_full += c->h_w_node[j];
    c->invA_full = 1.0 / ((double)c->Nx * c->Ly_full);
    c->meanFx_A = 0.0;
    if (cfg.F0 != 0.0) {
        for (int j = 0; j < Ny; ++j) {
            const double arg = (double)cfg.nforce * kPiD * ((c->h_y[j] + cfg.h) / (2.0 * cfg.h));
            c->meanFx_A += cfg.F0 * std::sin(arg) * c->h_w_node[j];
        }
        c->meanFx_A /= c->Ly_full;
    }
    c->psi_bot = 0.0; c->psi_top = 2.0 * cfg.h * cfg.Ub;
    c->closure_diag = cfg.closure_diag != 0;

    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (c->num_sms <= 0) c->num_sms = 148;

    c->thomas_groups = (c->H + 15) / 16;
    auto fail = [&]() { context_destroy(c); return -1; };
    RowTables& rt = c->rt;
    if (dalloc(&rt.y, Ny) || dalloc(&rt.a_node, Ny) || dalloc(&rt.a_edge, Ny) || dalloc(&rt.dy_edge, Ny) ||
        dalloc(&rt.w_node, Ny) || dalloc(&rt.wt_node, Ny) || dalloc(&rt.frow, Ny) || dalloc(&rt.st_cj, Ny) ||
        dalloc(&rt.st_ap, Ny) || dalloc(&rt.st_am, Ny) || dalloc(&rt.asub, Ny) ||
        dalloc(&rt.csup, Ny) || dalloc(&rt.inv_csup, Ny))
        return fail();
    if (cfg.mms) {
        if (dalloc(&rt.mms_g, Ny) || dalloc(&rt.mms_gpp, Ny) || dalloc(&rt.mms_sin2, Ny) ||
            dalloc(&rt.mms_sk, c->Nx) || dalloc(&rt.mms_s2k, c->Nx))
            return fail();
    }
    if (dalloc(&c->w, c->N) || dalloc(&c->w1, c->N) || dalloc(&c->w2, c->N) || dalloc(&c->psi, c->N) ||
        dalloc(&c->rhs, c->N) || dalloc(&c->J, c->N))
        return fail();
    if (dalloc(&c->hat, (size_t)Ny * c->Hp) || dalloc(&c->cp, (size_t)c->Ni * c->Hp) ||
        dalloc(&c->wN, (size_t)c->M + 1))
        return fail();
    c->thomas_nseg = (c->Ni + TS_ROWS - 1) / TS_ROWS;
    c->thomas_nsb = (c->thomas_nseg + TS_NW - 1) / TS_NW;
    if (dalloc(&c->tconst, (size_t)c->thomas_nseg * 3 * c->Hp) || dalloc(&c->tmaps, (size_t)c->thomas_nseg * 4 * c->Hp) ||
        dalloc(&c->tblk, (size_t)c->thomas_groups * c->thomas_nsb * 5 * 32) ||
        dalloc(&c->tbcarry, (size_t)c->thomas_groups * c->thomas_nsb * 2 * 32))
        return fail();
    if (cudaMalloc((void**)&c->tcount, sizeof(unsigned int) * c->thomas_groups) != cudaSuccess ||
        cudaMemset(c->tcount, 0, sizeof(unsigned int) * c->thomas_groups) != cudaSuccess) {
        set_error("cudaMalloc of the Thomas counters failed");
        return fail();
    }
    // one buffer for the block partials of the max reduction (3 per block) and the per-row
    // partials of the diagnostics (32 per row); never reallocated (graphs keep its address)
    c->red_nblocks = 2 * c->num_sms;
    c->red_capacity = std::max((size_t)c->red_nblocks * 3, (size_t)Ny * 32);
    if (dalloc(&c->red_blocks, c->red_capacity) || dalloc(&c->red_out, 64)) return fail();
    if (dalloc(&c->ctl, 1)) return fail();
    if (cudaMallocHost((void**)&c->h_ctl, sizeof(Ctl)) != cudaSuccess) { set_error("cudaMallocHost failed"); return fail(); }

    auto H2D = [&](double* d, const std::vector<double>& h) {
        return cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    };
    if (H2D(rt.y, c->h_y) || H2D(rt.a_node, c->h_a_node) || H2D(rt.a_edge, c->h_a_edge) ||
        H2D(rt.dy_edge, c->h_dy_edge) || H2D(rt.w_node, c->h_w_node)) {
        set_error("metric upload failed");
        return fail();
    }
    std::vector<cpx<double>> tw_full, tw, wN;
    twiddles(c->M, tw_full, wN);
    p16_twiddle_table(c->M, tw_full.data(), tw);
    if (dalloc(&c->tw, tw.size())) return fail();
    if (cudaMemcpy(c->tw, tw.data(), tw.size() * sizeof(tw[0]), cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->wN, wN.data(), wN.size() * sizeof(wN[0]), cudaMemcpyHostToDevice)) {
        set_error("twiddle upload failed");
        return fail();
    }
    const double mms_k = 2.0 * kPiD * (double)cfg.mms_kx / cfg.Lx;
    const double mms_c = kPiD / (2.0 * cfg.h);
    k_setup_rows<<<(Ny + 127) / 128, 128>>>(rt, Ny, c->inv_deta2, c->deta, cfg.F0, cfg.nforce, cfg.h, mms_k, mms_c,
                                            0.25 * c->inv_dx * c->inv_deta, c->nu);
    if (cfg.mms) k_setup_mms_cols<<<(c->Nx + 127) / 128, 128>>>(rt.mms_sk, rt.mms_s2k, c->Nx, c->dx, mms_k);
    k_setup_cp<<<(c->H + 127) / 128, 128>>>(c->cp, rt.a_node, rt.a_edge, c->Nx, Ny, c->Hp, c->H, cfg.Lx, c->inv_deta2);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        set_error("setup kernels failed: %s", cudaGetErrorString(cudaGetLastError()));
        return fail();
    }
    if (cudaFuncSetAttribute(k_thomas_maps<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)thomas_smem_bytes()) ||
        cudaFuncSetAttribute(k_thomas_apply<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)thomas_smem_bytes()) ||
        cudaFuncSetAttribute(k_thomas_maps<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)thomas_smem_bytes()) ||
        cudaFuncSetAttribute(k_thomas_apply<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)thomas_smem_bytes())) {
        set_error("cudaFuncSetAttribute (Thomas shared memory) failed: %s", cudaGetErrorString(cudaGetLastError()));
        return fail();
    }
    {
        ThomasParams tp = thomas_params(c);
        dim3 grid((c->Hp + 127) / 128, c->thomas_nseg);
        k_thomas_consts<<<grid, 128>>>(tp);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
            set_error("Thomas table setup failed: %s", cudaGetErrorString(cudaGetLastError()));
            return fail();
        }
    }
    // one-pass cluster solve when a cluster of at most 8 CTAs holds every interior row in
    // registers (at most 32 x 16 rows per CTA) and such clusters can be resident; otherwise the
    // two-pass form
    {
        int L = 1;
        while (TC_NSEG * L < (c->Ni + TC_MAX_CLUSTER - 1) / TC_MAX_CLUSTER) L *= 2;
        const int R = TC_NSEG * L, C = (c->Ni + R - 1) / R;
        const size_t smem = tc_smem_bytes(R);
        ThomasClusterKernel kern = thomas_cluster_kernel(L);
        int max_smem = 0;
        cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (kern && C <= TC_MAX_CLUSTER && smem + 4096 <= (size_t)max_smem &&
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
            encode_field_map(&c->tm_hat, reinterpret_cast<const double*>(c->hat), 2 * c->Hp, Ny, 2 * TC_KX,
                             std::min(R, TC_BOX)) == 0 &&
            encode_field_map(&c->tm_cp, c->cp, c->Hp, c->Ni, TC_KX, std::min(R, TC_BOX)) == 0) {
            cudaLaunchConfig_t lc{};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
            lc.gridDim = dim3(C * (c->Hp / TC_KX));
            lc.blockDim = dim3(TC_THREADS);
            lc.dynamicSmemBytes = smem;
            lc.attrs = at; lc.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &lc) == cudaSuccess && nclusters > 0) {
                c->thomas_cluster = true;
                c->thomas_cluster_ok = true;
                c->tc_cluster = C;
                c->tc_L = L;
                c->tc_smem = smem;
                c->tc_nclusters = std::min(nclusters, c->Hp / TC_KX);
            }
        }
        cudaGetLastError();                         // a refused attribute or query only selects the two passes
    }
    {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_maxuv_dt<true>, 256, 0) != cudaSuccess || per_sm < 1) {
            set_error("k_maxuv_dt cannot be resident: %s", cudaGetErrorString(cudaGetLastError()));
            return fail();
        }
        c->maxuv_ctas = per_sm * c->num_sms;
    }
    // stage kernel: persistent TMA variant when every tile row holds two or more tiles
    c->stage_tma = c->stage_tma_ok = (c->Nx >= 2 * ST_TX);
    c->rowfft_pf = c->rowfft_pf_ok = (c->M == 16 * IP_NT);
    if (c->rowfft_pf_ok) {
        // arrival counters of the band boundaries of the inverse transform (at most Ny / 2 bands)
        const size_t nb = (size_t)Ny / 2 + 2;
        if (cudaMalloc((void**)&c->bcount, nb * sizeof(unsigned)) != cudaSuccess ||
            cudaMemset(c->bcount, 0, nb * sizeof(unsigned)) != cudaSuccess) {
            set_error("cudaMalloc of the band counters failed");
            return fail();
        }
    }
    if (c->stage_tma) {
        if (encode_field_map(&c->tm_psi, c->psi, c->Nx, Ny) || encode_field_map(&c->tm_w[0], c->w, c->Nx, Ny) ||
            encode_field_map(&c->tm_w[1], c->w1, c->Nx, Ny) || encode_field_map(&c->tm_w[2], c->w2, c->Nx, Ny) ||
            encode_field_map(&c->tm_wn, c->w, c->Nx, Ny, ST_TX, ST_TY))
            return fail();
        int per_sm = 0;
        if (cudaFuncSetAttribute(k_stage_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_tma_smem_bytes()) ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_tma, 256, stage_tma_smem_bytes()) ||
            per_sm < 1) {
            set_error("k_stage_tma cannot be resident: %s", cudaGetErrorString(cudaGetLastError()));
            return fail();
        }
        const int ntiles = (c->Nx / ST_TX) * ((Ny + ST_TY - 1) / ST_TY);
        c->stage_tma_grid = std::min(ntiles, per_sm * c->num_sms);
    }
    if (cfg.precision == 32) {
        c->prec32 = true;
        if (setup32(c)) return fail();
        // the cluster solve over the FP32 spectral buffer (setup32 allocated it)
        if (c->thomas_cluster_ok) {
            const int R = TC_NSEG * c->tc_L, C = c->tc_cluster;
            const size_t smem = tc_smem_bytes(R, true);
            ThomasClusterKernel kern = thomas_cluster_kernel(c->tc_L, true);
            cudaLaunchConfig_t lc{};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
            lc.gridDim = dim3(C * (c->Hp / TC_KX));
            lc.blockDim = dim3(TC_THREADS);
            lc.dynamicSmemBytes = smem;
            lc.attrs = at; lc.numAttrs = 1;
            int nclusters = 0;
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
                encode_map_2d(&c->tm_hat32, c->hat32, true, 2 * c->Hp, Ny, 2 * TC_KX, std::min(R, TC_BOX)) != 0 ||
                cudaOccupancyMaxActiveClusters(&nclusters, kern, &lc) != cudaSuccess || nclusters < 1) {
                // the FP64 spectra's cluster form is resident, so this one (less shared memory) is too
                set_error("the FP32-spectra cluster solve cannot be set up: %s", cudaGetErrorString(cudaGetLastError()));
                return fail();
            }
            c->tc_smem32 = smem;
            c->tc_nclusters32 = std::min(nclusters, c->Hp / TC_KX);
        }
    }
    Ctl h{};
    h.t = 0.0; h.dt = cfg.dt_init; h.next_out = 1e300; h.next_snap = 1e300; h.next_diag = 1e300;
    if (cudaMemcpy(c->ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice) != cudaSuccess) { set_error("ctl upload"); return fail(); }
    *out = c;
    return 0;
}

void context_destroy(Context* c) {
    if (!c) return;
    RowTables& rt = c->rt;
    for (double* p : {rt.y, rt.a_node, rt.a_edge, rt.dy_edge, rt.w_node, rt.wt_node, rt.frow, rt.st_cj, rt.st_ap, rt.st_am, rt.asub, rt.csup,
                      rt.inv_csup, rt.mms_g, rt.mms_gpp, rt.mms_sin2, rt.mms_sk, rt.mms_s2k, c->w, c->w1, c->w2,
                      c->psi, c->rhs, c->J, c->cp, c->red_blocks, c->red_out})
        if (p) cudaFree(p);
    if (c->closure_tau) cudaFree(c->closure_tau);
    if (c->hat) cudaFree(c->hat);
    if (c->tconst) cudaFree(c->tconst);
    if (c->tmaps) cudaFree(c->tmaps);
    if (c->tblk) cudaFree(c->tblk);
    if (c->tbcarry) cudaFree(c->tbcarry);
    if (c->tcount) cudaFree(c->tcount);
    if (c->tw) cudaFree(c->tw);
    if (c->wN) cudaFree(c->wN);
    if (c->ctl) cudaFree(c->ctl);
    if (c->h_ctl) cudaFreeHost(c->h_ctl);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->run_exec) cudaGraphExecDestroy(c->run_exec);
    destroy32(c);
    if (c->spec_acc) cudaFree(c->spec_acc);
    if (c->moments) cudaFree(c->moments);
    if (c->stats_acc) cudaFree(c->stats_acc);
    if (c->bcount) cudaFree(c->bcount);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    delete c;
}

// The max reduction of an adaptive FP64 step runs in its stage-3 inverse transform when that is the
// prefetching form (k_ifft_thom_pf); the stage-1 kernel then takes dt from the maxima it left.
static bool fused_max(const Context* c) { return c->cfg.adapt && !c->prec32 && c->rowfft_pf && c->max_fused; }

// ---- launchers ----
static StageParams stage_params(Context* c) {
    StageParams p{};
    p.psi = c->psi; p.rt = c->rt; p.ctl = c->ctl;
    p.Nx = c->Nx; p.Ny = c->Ny; p.mms = c->cfg.mms;
    p.inv_dx = c->inv_dx; p.inv_deta = c->inv_deta; p.inv_dx2 = c->inv_dx2; p.inv_deta2 = c->inv_deta2;
    p.nu = c->nu; p.lin_drag = c->cfg.lin_drag;
    p.mms_A0 = c->cfg.mms_A0; p.mms_eps = c->cfg.mms_eps; p.mms_Om = c->cfg.mms_Om;
    p.mms_k = 2.0 * kPiD * (double)c->cfg.mms_kx / c->cfg.Lx; p.mms_c = kPiD / (2.0 * c->cfg.h);
    p.dt_from_max = fused_max(c) ? 1 : 0;
    p.cfl = c->cfg.cfl; p.cvisc = c->cfg.cvisc; p.dx = c->dx; p.deta = c->deta; p.inv_dymin2 = c->inv_dymin2;
    p.dt_max = c->cfg.dt_max;
    return p;
}

int launch_stage(Context* c, int stage, const double* w_in, const double* w_n, double* w_out, cudaStream_t s,
                 double* rhs_out) {
    StageParams p = stage_params(c);
    p.w_in = w_in; p.w_n = w_n; p.w_out = w_out; p.rhs_out = rhs_out; p.stage = stage;
    // the learned closure's tau of this stage's state (the model runs just before the stage)
    if (c->closure_net) {
        if (stage == 1 || c->closure_every_stage) {
            double* u = c->closure_tau + c->N;
            double* v = c->closure_tau + 2 * c->N;
            if (uv_from_psi(c, c->psi, u, v, s) || cnn_forward(c->closure_net, w_in, c->psi, u, v, c->closure_tau, s))
                return -1;
        }
        p.closure = c->closure_tau;
    }
    if (c->stage_tma) {
        if (stage > 1 && w_n != c->w) { set_error("launch_stage: omega^n is not the context's omega"); return -1; }
        StageMaps maps;
        maps.psi = c->tm_psi;
        maps.wn = c->tm_wn;
        if (w_in == c->w) maps.w = c->tm_w[0];
        else if (w_in == c->w1) maps.w = c->tm_w[1];
        else if (w_in == c->w2) maps.w = c->tm_w[2];
        else { set_error("launch_stage: omega^(s) is not a context buffer"); return -1; }
        return launch_step_kernel(c, k_stage_tma, dim3(c->stage_tma_grid), dim3(256), stage_tma_smem_bytes(), s, nullptr,
                                  maps, p);
    }
    const dim3 grid((c->Nx + ST_TX - 1) / ST_TX, (c->Ny + ST_TY - 1) / ST_TY);
    return launch_step_kernel(c, k_stage, grid, dim3(256), 0, s, nullptr, p);
}

static size_t fft_smem(int M) { return fft_smem_bytes(M); }

static FftParams fft_params(Context* c) {
    FftParams p{};
    p.a_node = c->rt.a_node; p.bcount = c->bcount; p.inv_dx = c->inv_dx; p.inv_deta = c->inv_deta;
    p.hat = c->hat; p.tw = c->tw; p.wN = c->wN; p.Nx = c->Nx; p.Ny = c->Ny; p.Hp = c->Hp;
    p.dy_edge = c->rt.dy_edge; p.w_node = c->rt.w_node; p.ctl = c->ctl; p.free_slip = c->cfg.free_slip;
    p.psi_bot = c->psi_bot; p.psi_top = c->psi_top; p.invA_full = c->invA_full;
    return p;
}

// Forward transforms: one row per CTA (many small CTAs per SM hide each other's load latency).
// Row transforms: one wave of CTAs (occupancy x SMs, at most the number of rows), each taking
// the rows blockIdx.x, blockIdx.x + grid, ...; a partial second wave of one-row CTAs would
// leave most SMs idle at its end.
template <typename K> static int fft_wave(K kern, size_t smem, int nrows, int num_sms, int* grid) {
    int per_sm = 0;
    NSE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    NSE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, IP_NT, smem));
    if (per_sm < 1) { set_error("a row transform kernel cannot be resident (%zu bytes of shared memory)", smem); return -1; }
    *grid = std::max(1, std::min(nrows, per_sm * num_sms));
    return 0;
}

template <int M> static int fft_fwd_t(Context* c, FftParams& p, cudaStream_t s) {
    if constexpr (M == 16 * IP_NT) if (c->rowfft_pf) {
        // the real rows prefetched into shared memory by bulk copies (k_fft_fwd_pf)
        const size_t sm = FftPf<M>::smem;
        int grid = 0;
        if (fft_wave(k_fft_fwd_pf<M>, sm, p.nrows, c->num_sms, &grid)) return -1;
        return launch_step_kernel(c, k_fft_fwd_pf<M>, dim3(grid), dim3(IP_NT), sm, s, nullptr, p);
    }
    const size_t sm = fft_smem(M);
    int grid = 0;
    if (fft_wave(k_fft_fwd<M>, sm, p.nrows, c->num_sms, &grid)) return -1;
    return launch_step_kernel(c, k_fft_fwd<M>, dim3(grid), dim3(IP_NT), sm, s, nullptr, p);
}

// Inverse transforms: one wave of CTAs over contiguous bands of floor or ceil(Ny / wave) rows
// (adjacent rows of the spectral buffer are adjacent in memory; strided rows measured slower).
// The Thom closure is applied by the CTA that writes the second row of each wall.
template <int M> static int fft_inv_t(Context* c, FftParams& p, cudaStream_t s) {
    if constexpr (M == 16 * IP_NT) if (c->rowfft_pf) {
        // the spectral rows prefetched into shared memory by bulk copies (k_ifft_thom_pf)
        // bands of two or more rows (the fused max reduction pairs the rows at band boundaries)
        const size_t sm = IfftPf<M>::smem;
        int wave = 0;
        if (fft_wave(k_ifft_thom_pf<M>, sm, c->Ny, c->num_sms, &wave)) return -1;
        return launch_step_kernel(c, k_ifft_thom_pf<M>, dim3(std::max(1, std::min(wave, c->Ny / 2))), dim3(IP_NT), sm, s,
                                  nullptr, p);
    }
    const size_t sm = fft_smem(M);
    int wave = 0;
    if (fft_wave(k_ifft_thom<M>, sm, c->Ny, c->num_sms, &wave)) return -1;
    const int grid = std::max(1, std::min(wave, c->Ny));           // bands of Ny / grid rows (even split)
    return launch_step_kernel(c, k_ifft_thom<M>, dim3(grid), dim3(IP_NT), sm, s, nullptr, p);
}

#define NSE_FFT_DISPATCH(FN)                                                       \
    switch (c->M) {                                                                \
        case 2: return FN<2>(c, p, s);       case 4: return FN<4>(c, p, s);        \
        case 8: return FN<8>(c, p, s);       case 16: return FN<16>(c, p, s);      \
        case 32: return FN<32>(c, p, s);     case 64: return FN<64>(c, p, s);      \
        case 128: return FN<128>(c, p, s);   case 256: return FN<256>(c, p, s);    \
        case 512: return FN<512>(c, p, s);   case 1024: return FN<1024>(c, p, s);  \
        case 2048: return FN<2048>(c, p, s); case 4096: return FN<4096>(c, p, s);  \
        case 8192: return FN<8192>(c, p, s);                                       \
        default: set_error("no FFT kernel for M = %d", c->M); return -1;           \
    }

int launch_fft_fwd(Context* c, const double* src, cudaStream_t s) {
    if (reinterpret_cast<uintptr_t>(src) % 16 != 0) {
        set_error("omega must be 16-byte aligned for the row transform (got %p)", (const void*)src);
        return -1;
    }
    FftParams p = fft_params(c);
    p.src = src;
    p.row0 = 1;
    p.nrows = c->Ni;
    NSE_FFT_DISPATCH(fft_fwd_t)
}

// Forward transform of every row 0..Ny-1 of src into the spectral buffer (1-D spectra).
int launch_fft_all_rows(Context* c, const double* src, cudaStream_t s) {
    if (reinterpret_cast<uintptr_t>(src) % 16 != 0) {
        set_error("the field must be 16-byte aligned for the row transform (got %p)", (const void*)src);
        return -1;
    }
    FftParams p = fft_params(c);
    p.src = src;
    p.row0 = 0;
    p.nrows = c->Ny;
    NSE_FFT_DISPATCH(fft_fwd_t)
}

int launch_ifft_thom(Context* c, double* psi, double* w, int stage, bool do_thom, bool closure, cudaStream_t s,
                     bool advance) {
    FftParams p = fft_params(c);
    p.psi = psi; p.w = w; p.stage = stage; p.do_thom = do_thom ? 1 : 0; p.closure = closure ? 1 : 0;
    p.advance = advance ? 1 : 0;
    p.fuse_max = (advance && fused_max(c)) ? 1 : 0;
    NSE_FFT_DISPATCH(fft_inv_t)
}

// The two passes of the segmented Thomas solve: the segment maps (and, in the last CTA of each
// column group, the carries), then the rerun of every segment from its carries.
int launch_thomas_maps(Context* c, cudaStream_t s, bool homog) {
    return launch_step_kernel(c, homog ? k_thomas_maps<true> : k_thomas_maps<false>,
                              dim3(c->thomas_groups * c->thomas_nsb), dim3(TS_NW * 32),
                              thomas_smem_bytes(), s, nullptr, thomas_params(c, homog));
}
int launch_thomas_apply(Context* c, cudaStream_t s, bool homog) {
    return launch_step_kernel(c, homog ? k_thomas_apply<true> : k_thomas_apply<false>,
                              dim3(c->thomas_groups * c->thomas_nsb), dim3(TS_NW * 32),
                              thomas_smem_bytes(), s, nullptr, thomas_params(c, homog));
}
// The one-pass form: one cluster of tc_cluster CTAs per 8-kx column group.
int launch_thomas_cluster(Context* c, cudaStream_t s, bool homog) {
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = c->tc_cluster; at.val.clusterDim.y = 1; at.val.clusterDim.z = 1;
    ThomasMaps maps;
    maps.hat = homog ? c->tm_hat32 : c->tm_hat;
    maps.cp = c->tm_cp;
    // persistent: the resident clusters
    const int ncl = homog ? c->tc_nclusters32 : c->tc_nclusters;
    return launch_step_kernel(c, thomas_cluster_kernel(c->tc_L, homog), dim3(c->tc_cluster * ncl), dim3(TC_THREADS),
                              homog ? c->tc_smem32 : c->tc_smem, s, &at, maps, thomas_params(c, homog));
}

// The kernel forms of the step (each falls back to the one the context can use); drops the
// captured graphs when anything changes.
PlanForms get_plan(const Context* c) {
    return PlanForms{c->prec32 ? c->stage32_tma : c->stage_tma, c->thomas_cluster, c->rowfft_pf, fused_max(c), c->pdl};
}

int set_plan(Context* c, const PlanForms& f) {
    const bool st = f.stage_tma && (c->prec32 ? c->stage32_tma_ok : c->stage_tma_ok);
    const bool pf = f.rowfft_pf && c->rowfft_pf_ok;
    const bool cur = c->prec32 ? c->stage32_tma : c->stage_tma;
    const bool fused_before = fused_max(c);
    const bool fused_after = c->cfg.adapt && !c->prec32 && pf && f.max_fused;
    const bool pdl = f.pdl;
    if (st != cur || pf != c->rowfft_pf || fused_before != fused_after || pdl != c->pdl) {
        NSE_CUDA_TRY(cudaDeviceSynchronize());
        if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
        if (c->run_exec) { cudaGraphExecDestroy(c->run_exec); c->run_exec = nullptr; }
        if (c->prec32) c->stage32_tma = st; else c->stage_tma = st;
        c->rowfft_pf = pf;
        c->pdl = pdl;
    }
    c->max_fused = f.max_fused;
    if (set_tridiag_form(c, f.clusters)) return -1;
    // the next step may take its dt from the maxima of the current psi
    if (refresh_maxima(c, 0)) return -1;
    NSE_CUDA_TRY(cudaDeviceSynchronize());
    return 0;
}

int set_tridiag_form(Context* c, bool clusters) {
    const bool use = clusters && c->thomas_cluster_ok;
    if (use == c->thomas_cluster) return 0;
    // the captured graphs hold the other form's kernels: wait for any launch of them, then drop
    // them (they are captured again at the next step)
    NSE_CUDA_TRY(cudaDeviceSynchronize());
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
    if (c->run_exec) { cudaGraphExecDestroy(c->run_exec); c->run_exec = nullptr; }
    c->thomas_cluster = use;
    return 0;
}

// Launches of one tridiagonal solve: 1 (cluster form) or 2 (maps, apply); part i of them.
int thomas_launches(const Context* c) { return c->thomas_cluster ? 1 : 2; }
const char* thomas_kernel_name(const Context* c, int i) {
    if (c->thomas_cluster) return "k_thomas_cluster";
    return i == 0 ? "k_thomas_maps" : "k_thomas_apply";
}
int launch_thomas_part(Context* c, int i, cudaStream_t s, bool homog) {
    if (c->thomas_cluster) return launch_thomas_cluster(c, s, homog);
    return i == 0 ? launch_thomas_maps(c, s, homog) : launch_thomas_apply(c, s, homog);
}
int launch_thomas(Context* c, cudaStream_t s) {
    for (int i = 0; i < thomas_launches(c); ++i)
        if (launch_thomas_part(c, i, s, false)) return -1;
    return 0;
}

// the reference's standalone Thom launcher (src/ops.cu:270-276)
int launch_thom(Context* c, double* w, const double* psi, cudaStream_t s) {
    ThomParams p{};
    p.w = w; p.psi = psi; p.dy_edge = c->rt.dy_edge; p.Nx = c->Nx; p.Ny = c->Ny; p.free_slip = c->cfg.free_slip;
    p.psi_bot = c->psi_bot; p.psi_top = c->psi_top;
    k_thom<<<(c->Nx + 255) / 256, 256, 0, s>>>(p);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_maxuv(Context* c, const double* psi, bool set_dt, cudaStream_t s, bool next_only) {
    MaxParams p{};
    p.psi = psi; p.a_node = c->rt.a_node; p.ctl = c->ctl; p.next_only = next_only ? 1 : 0;
    p.Nx = c->Nx; p.Ny = c->Ny; p.adapt = c->cfg.adapt; p.set_dt = set_dt ? 1 : 0;
    p.inv_dx = c->inv_dx; p.inv_deta = c->inv_deta; p.cfl = c->cfg.cfl; p.cvisc = c->cfg.cvisc;
    p.dx = c->dx; p.deta = c->deta; p.nu = c->nu; p.inv_dx2 = c->inv_dx2; p.inv_dymin2 = c->inv_dymin2;
    p.dt_max = c->cfg.dt_max;
    int grid = 1;
    maxuv_plan(p, c->maxuv_ctas, c->maxuv_ctas, grid);
    return launch_step_kernel(c, k_maxuv_dt<true>, dim3(grid), dim3(256), 0, s, nullptr, p);
}

// Poisson solve of the reference (src/poisson.cuh:83-118): omega -> psi.
int poisson_solve(Context* c, const double* w, double* psi, cudaStream_t s) {
    if (launch_fft_fwd(c, w, s)) return -1;
    if (launch_thomas(c, s)) return -1;
    if (launch_ifft_thom(c, psi, nullptr, 0, false, false, s)) return -1;
    return 0;
}

// One SSPRK(3,3) step (src/main.cu:439-541) with dt from the control block. With ev != nullptr
// an event is recorded before the step and after every kernel (for per-kernel timing).
static int step_impl(Context* c, cudaStream_t s, bool store_rhs, cudaEvent_t* ev) {
    if (c->prec32) return step32_impl(c, s, store_rhs, ev);
    int k = 0;
    auto mark = [&]() -> int {
        if (ev) NSE_CUDA_TRY(cudaEventRecord(ev[k++], s));
        return 0;
    };
    if (mark()) return -1;
    if (c->cfg.adapt && !fused_max(c)) {
        if (launch_maxuv(c, c->psi, true, s) || mark()) return -1;
    }
    double* wst[3] = {c->w1, c->w2, c->w};
    const double* win[3] = {c->w, c->w1, c->w2};
    for (int st = 1; st <= 3; ++st) {
        if (launch_stage(c, st, win[st - 1], c->w, wst[st - 1], s, (store_rhs && st == 3) ? c->rhs : nullptr) || mark())
            return -1;
        if (launch_fft_fwd(c, wst[st - 1], s) || mark()) return -1;
        for (int i = 0; i < thomas_launches(c); ++i)
            if (launch_thomas_part(c, i, s, false) || mark()) return -1;
        // the stage-3 transform also advances the time (its last CTA)
        if (launch_ifft_thom(c, c->psi, wst[st - 1], st, true, c->closure_diag, s, st == 3) || mark()) return -1;
    }
    return 0;
}

int enqueue_step(Context* c, cudaStream_t s, bool store_rhs) { return step_impl(c, s, store_rhs, nullptr); }
int enqueue_step_timed(Context* c, cudaStream_t s, cudaEvent_t* ev, bool store_rhs) {
    return step_impl(c, s, store_rhs, ev);
}

// Names of the kernels of one step, in launch order (for the timed step).
const char* step_kernel_name(const Context* c, int k) {
    if (c->prec32) return step32_kernel_name(c, k);
    if (c->cfg.adapt && !fused_max(c)) {
        if (k == 0) return "k_maxuv_dt";
        --k;
    }
    const int per = 3 + thomas_launches(c);
    if (k < 0 || k >= 3 * per) return "";
    const int i = k % per;
    if (i == 0) return c->stage_tma ? "k_stage_tma" : "k_stage";
    if (i == 1) return "k_fft_fwd";
    if (i == per - 1) return "k_ifft_thom";
    return thomas_kernel_name(c, i - 2);
}

int launches_per_step(const Context* c) {
    if (c->prec32) return (c->cfg.adapt ? 1 : 0) + 3 * (3 + thomas_launches(c));
    return (c->cfg.adapt && !fused_max(c) ? 1 : 0) + 3 * (3 + thomas_launches(c));
}

// max |u|, |v|, |v| a of the current psi into the control block (also as the next step's maxima):
// after the state is set, or the kernel plan changes.
int refresh_maxima(Context* c, cudaStream_t s) {
    if (c->prec32 || !c->cfg.adapt) return 0;
    return launch_maxuv(c, c->psi, false, s, true);
}

// nsteps steps; with use_graph the step is captured once into a CUDA graph and replayed.
int run_steps(Context* c, int nsteps, bool use_graph, cudaStream_t s, bool store_rhs) {
    if (nsteps <= 0) return 0;
    if (!use_graph || store_rhs) {
        for (int i = 0; i < nsteps; ++i)
            if (enqueue_step(c, s, store_rhs && i == nsteps - 1)) return -1;
        return 0;
    }
    if (!c->graph_exec) {
        if (!c->cap_stream) NSE_CUDA_TRY(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
        NSE_CUDA_TRY(cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_step(c, c->cap_stream, false);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c->cap_stream, &g);
        if (rc != 0) { if (g) cudaGraphDestroy(g); return -1; }
        NSE_CUDA_TRY(e);
        const cudaError_t e2 = cudaGraphInstantiate(&c->graph_exec, g, 0);
        cudaGraphDestroy(g);
        NSE_CUDA_TRY(e2);
    }
    for (int i = 0; i < nsteps; ++i) NSE_CUDA_TRY(cudaGraphLaunch(c->graph_exec, s));
    return 0;
}

// Last node of the run loop's body: keep looping while no halt was requested and the step
// budget lasts (the budget bounds the device loop whatever the schedule says).
static __global__ void k_loop_cond(Ctl* ctl, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    ctl->run_budget -= 1;
    if (!ctl->halt && ctl->run_budget <= 0) {
        ctl->halt = 1;
        ctl->halt_reason |= 16;
    }
    cudaGraphSetConditional(h, ctl->halt ? 0u : 1u);
}

// Steps on the device until advance_time or the budget requests a halt: one graph launch holds
// a WHILE node whose body is one captured step followed by k_loop_cond. The run fields of the
// control block must be set (run = 1, halt = 0, run_budget > 0) before the launch.
int run_until_halt(Context* c, cudaStream_t s) {
    if (!c->run_exec) {
        if (!c->cap_stream) NSE_CUDA_TRY(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        NSE_CUDA_TRY(cudaGraphCreate(&g, 0));
        auto fail = [&](const char* what, cudaError_t e) {
            set_error("run graph: %s: %s", what, cudaGetErrorString(e));
            cudaGraphDestroy(g);
            return -1;
        };
        cudaGraphConditionalHandle h;
        cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) return fail("conditional handle", e);
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
        if (e != cudaSuccess) return fail("conditional node", e);
        cudaGraph_t body = np.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(c->cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail("capture", e);
        // the step stores its stage-3 rhs, which the diagnostics row after a run pairs with omega
        int rc = enqueue_step(c, c->cap_stream, true);
        if (rc == 0 && c->stats_dev) rc = enqueue_stats(c, c->cap_stream);
        if (rc == 0) k_loop_cond<<<1, 32, 0, c->cap_stream>>>(c->ctl, h);
        cudaGraph_t captured = nullptr;
        e = cudaStreamEndCapture(c->cap_stream, &captured);
        if (rc != 0) { cudaGraphDestroy(g); return -1; }
        if (e != cudaSuccess) return fail("end capture", e);
        e = cudaGraphInstantiate(&c->run_exec, g, 0);
        cudaGraphDestroy(g);
        NSE_CUDA_TRY(e);
    }
    NSE_CUDA_TRY(cudaGraphLaunch(c->run_exec, s));
    return 0;
}

// omega (device) -> initial solve + Thom, t = 0 (src/main.cu:197-215)
int set_initial_omega(Context* c, cudaStream_t s) {
    if (poisson_solve(c, c->w, c->psi, s)) return -1;
    if (launch_thom(c, c->w, c->psi, s)) return -1;
    if (c->prec32 && split32(c, s)) return -1;
    Ctl h{};
    h.t = 0.0; h.dt = c->cfg.dt_init; h.next_out = 1e300; h.next_snap = 1e300; h.next_diag = 1e300;
    NSE_CUDA_TRY(cudaMemcpyAsync(c->ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    if (refresh_maxima(c, s)) return -1;
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

}  // namespace nse2d
