// The reference's driver-side C++ API on this library (include/nse2d/*.hpp): build_y_metrics,
// the operator launchers of src/ops.cuh:12-81, the diagnostic launchers of src/diag.cuh:12-113,
// Spectra1D (src/diag.cuh:123-191) and Poisson2D_Z2Z (src/poisson.cuh:18-119). Written for this
// project. These serve code written against the reference's API; the time step itself runs on the
// fused kernels of step_kernels.cuh.
//
// Each operator restates the reference's per-point formula (cited per kernel). The sums follow the
// reference's semantics: the launcher zeroes its device scalars, and every CTA adds its partial sum
// with atomicAdd (so results agree with the reference's to round-off, not to the bit). No static
// scratch: the one launcher that used some in the reference (the enstrophy balance's Laplacian)
// evaluates the stencil inside its reduction, and the maxima are combined by atomic maxima on the
// bit patterns of the caller's (non-negative) output scalars.
#include <cmath>
#include <stdexcept>
#include <string>

#include "nse2d_internal.h"
#include "step_kernels.cuh"
#include "../../include/nse2d.h"
#include "../../include/nse2d/diag.hpp"
#include "../../include/nse2d/poisson.hpp"
#include "../host/snapshot.h"

namespace nse2d {
namespace {

constexpr int kRedThreads = 256;

__device__ __forceinline__ int wrap_x(int i, int Nx) { return i < 0 ? i + Nx : (i >= Nx ? i - Nx : i); }

// forcing profile of the vorticity equation: f = -F0 (n pi / 2h) cos(n pi (y + h) / 2h)
__device__ __forceinline__ double f_omega(double y, double h, double F0, int nforce) {
    const double arg = (double)nforce * kPiD * ((y + h) / (2.0 * h));
    return -F0 * ((double)nforce * kPiD / (2.0 * h)) * cos(arg);
}

// ---- elementwise operators ----
// mapped Laplacian, walls 0: src/ops.cu:471-499
__global__ void k_laplacian(const double* __restrict__ q, double* __restrict__ out, int Nx, int Ny, double inv_dx2,
                            double inv_deta2, const double* __restrict__ a_node, const double* __restrict__ a_edge) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny) return;
    const size_t c = (size_t)iy * Nx + ix;
    if (iy == 0 || iy == Ny - 1) { out[c] = 0.0; return; }
    const double* r = q + (size_t)iy * Nx;
    const double dxx = (r[wrap_x(ix + 1, Nx)] - 2 * r[ix] + r[wrap_x(ix - 1, Nx)]) * inv_dx2;
    const double dyy = a_node[iy] * (a_edge[iy] * (q[c + Nx] - q[c]) - a_edge[iy - 1] * (q[c] - q[c - Nx])) * inv_deta2;
    out[c] = dxx + dyy;
}

// rhs = -J + nu lap + f(y) - r omega: src/ops.cu:515-534
__global__ void k_rhs(const double* __restrict__ J, const double* __restrict__ lap, const double* __restrict__ omg,
                      double* __restrict__ rhs, int Nx, int Ny, double nu, double F0, int nforce, double h,
                      double drag, const double* __restrict__ y) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny) return;
    const size_t c = (size_t)iy * Nx + ix;
    const double f = (F0 != 0.0) ? f_omega(y[iy], h, F0, nforce) : 0.0;
    rhs[c] = -J[c] + nu * lap[c] + f - drag * omg[c];
}

// the manufactured forcing of src/ops.cu:559-626 added to rhs: omega_ex = A(t) sin(kx) g(y) with
// g = k^2 sin^2(theta) - 2 c^2 cos(2 theta), theta = c (y + h), c = pi / 2h, A = A0 (1 + eps sin(Om t));
// f = sin(kx) (A' g + nu A (k^2 g - g'') + r A g) - A^2 k c^3 sin(2kx) sin(2 theta)
__global__ void k_mms_add(double* __restrict__ rhs, int Nx, int Ny, double Lx, double h, double t, double nu, double r,
                          double A0, double eps, double Om, int kx_mode, const double* __restrict__ y) {
    const size_t N = (size_t)Nx * Ny;
    const double dx = Lx / (double)Nx, k = 2.0 * kPiD * (double)kx_mode / Lx, c = kPiD / (2.0 * h);
    const double A = A0 * (1.0 + eps * sin(Om * t)), Ap = A0 * (eps * Om * cos(Om * t));
    const double c2 = c * c, k2 = k * k;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / (size_t)Nx), i = (int)(idx - (size_t)j * Nx);
        const double th = c * (y[j] + h), sth = sin(th);
        const double cos2 = cos(2.0 * th), sin2 = sin(2.0 * th);
        const double g = k2 * (sth * sth) - 2.0 * c2 * cos2;
        const double gpp = 2.0 * c2 * cos2 * (k2 + 4.0 * c2);
        const double x = (double)i * dx;
        const double lin = Ap * g + (nu * A) * (k2 * g - gpp) + (r * A) * g;
        rhs[idx] += sin(k * x) * lin - (A * A) * k * (c2 * c) * sin(2.0 * k * x) * sin2;
    }
}

// the Shu-Osher combines: src/ops.cu:644-669
__global__ void k_axpy(double* y, const double* x, const double* r, double dt, size_t N) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) y[i] = x[i] + dt * r[i];
}
__global__ void k_ssprk2(double* w2, const double* w, const double* w1, const double* rhs, double dt, size_t N) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) w2[i] = 0.75 * w[i] + 0.25 * (w1[i] + dt * rhs[i]);
}
__global__ void k_ssprk3(double* wn, const double* w, const double* w2, const double* rhs, double dt, size_t N) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) wn[i] = (1.0 / 3.0) * w[i] + (2.0 / 3.0) * (w2[i] + dt * rhs[i]);
}

// ---- reductions: sum over the grid of two per-point terms, then atomic adds of CTA partials ----
template <class F>
__global__ void __launch_bounds__(kRedThreads) k_sum2(F f, int Nx, int Ny, double* o0, double* o1) {
    const size_t N = (size_t)Nx * Ny;
    double a = 0.0, b = 0.0;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / (size_t)Nx), i = (int)(idx - (size_t)j * Nx);
        f(i, j, a, b);
    }
    __shared__ double sa[kRedThreads / 32], sb[kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sa[warp] = a; sb[warp] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < kRedThreads / 32; ++w) { ta += sa[w]; tb += sb[w]; }
        atomicAdd(o0, ta);
        if (o1) atomicAdd(o1, tb);
    }
}

template <class F> void sum2(const char* what, F f, int Nx, int Ny, double* o0, double* o1, cudaStream_t s) {
    cudaMemsetAsync(o0, 0, sizeof(double), s);
    if (o1) cudaMemsetAsync(o1, 0, sizeof(double), s);
    const size_t N = (size_t)Nx * Ny;
    const int blocks = (int)std::min<size_t>(8192, (N + kRedThreads - 1) / kRedThreads);
    k_sum2<<<blocks < 1 ? 1 : blocks, kRedThreads, 0, s>>>(f, Nx, Ny, o0, o1);
    compat_check_launch(what);
}

// Omega and |grad omega|^2 on the interior rows, centred differences: src/diag.cu:6-38
struct EnstDiss {
    const double *w, *a_node, *w_node;
    int Nx;
    double inv_dx, inv_deta;
    int Ny;
    __device__ void operator()(int i, int j, double& s0, double& s1) const {
        if (j == 0 || j == Ny - 1) return;
        const double* r = w + (size_t)j * Nx;
        const double wc = r[i];
        const double wx = (r[wrap_x(i + 1, Nx)] - r[wrap_x(i - 1, Nx)]) * 0.5 * inv_dx;
        const double wy = a_node[j] * (r[i + Nx] - r[i - Nx]) * 0.5 * inv_deta;
        s0 += w_node[j] * (wc * wc);
        s1 += w_node[j] * (wx * wx + wy * wy);
    }
};

// the same over all rows, second-order one-sided eta differences at the walls: src/diag.cu:43-101
struct EnstDissFull {
    const double *w, *a_node, *w_node;
    int Nx, Ny;
    double inv_dx, inv_deta;
    __device__ void operator()(int i, int j, double& s0, double& s1) const {
        const double* r = w + (size_t)j * Nx;
        const double wc = r[i];
        const double wx = (r[wrap_x(i + 1, Nx)] - r[wrap_x(i - 1, Nx)]) * 0.5 * inv_dx;
        double we;
        if (j == 0) we = (-3.0 * wc + 4.0 * r[i + Nx] - 1.0 * r[i + 2 * (size_t)Nx]) * (0.5 * inv_deta);
        else if (j == Ny - 1) we = (3.0 * wc - 4.0 * r[i - Nx] + 1.0 * r[i - 2 * (size_t)Nx]) * (0.5 * inv_deta);
        else we = (r[i + Nx] - r[i - Nx]) * 0.5 * inv_deta;
        const double wy = a_node[j] * we;
        s0 += w_node[j] * (wc * wc);
        s1 += w_node[j] * (wx * wx + wy * wy);
    }
};

// summation-by-parts remainders eta_h, Phi_h of the mapped Laplacian: src/diag.cu:166-199
struct EnstSbp {
    const double *w, *a_edge, *wt_node;
    int Nx, Ny;
    double inv_dx, inv_deta;
    __device__ void operator()(int i, int j, double& s0, double& s1) const {
        const double* r = w + (size_t)j * Nx;
        const double w0 = r[i];
        if (j >= 1 && j <= Ny - 2) {
            const double d = (r[wrap_x(i + 1, Nx)] - w0) * inv_dx;
            s0 += wt_node[j] * d * d;
        }
        if (j <= Ny - 2) {
            const double d = r[i + Nx] - w0;
            s0 += a_edge[j] * d * d * inv_deta;
        }
        if (j == 0) s1 -= w0 * a_edge[0] * (r[i + Nx] - w0) * inv_deta;
        if (j == Ny - 1) s1 += w0 * a_edge[Ny - 2] * (w0 - r[i - Nx]) * inv_deta;
    }
};

// kinetic energy 0.5 (u^2 + v^2) on the interior rows: src/diag.cu:201-231
struct KineticEnergy {
    const double *psi, *a_node, *w_node;
    int Nx, Ny;
    double inv_dx, inv_deta;
    __device__ void operator()(int i, int j, double& s0, double&) const {
        if (j == 0 || j == Ny - 1) return;
        const double* r = psi + (size_t)j * Nx;
        const double u = (r[i + Nx] - r[i - Nx]) * 0.5 * inv_deta * a_node[j];
        const double v = -(r[wrap_x(i + 1, Nx)] - r[wrap_x(i - 1, Nx)]) * 0.5 * inv_dx;
        s0 += 0.5 * (u * u + v * v) * w_node[j];
    }
};

// |grad u|^2 + |grad v|^2 (u_y = -omega on the wall rows): src/diag.cu:250-348
struct EnergyDiss {
    const double *psi, *w, *a_node, *a_edge, *w_node;
    int Nx, Ny;
    double inv_dx, inv_deta;
    __device__ void operator()(int i, int j, double& s0, double&) const {
        const size_t c = (size_t)j * Nx + i;
        if (j == 0 || j == Ny - 1) {
            const double uy = -w[c];
            s0 += (uy * uy) * w_node[j];
            return;
        }
        const int ip = wrap_x(i + 1, Nx), im = wrap_x(i - 1, Nx);
        const double* r = psi + (size_t)j * Nx;
        const double* rp = r + Nx;
        const double* rm = r - Nx;
        const double a = a_node[j], ap = a_edge[j], am = a_edge[j - 1];
        const double pxp = (rp[ip] - rp[im]) * (0.5 * inv_dx), pxm = (rm[ip] - rm[im]) * (0.5 * inv_dx);
        const double ux = a * (pxp - pxm) * (0.5 * inv_deta);
        const double vy = -ux;
        const double vx = -(r[ip] - 2.0 * r[i] + r[im]) * (inv_dx * inv_dx);
        const double uy = a * (ap * (rp[i] - r[i]) - am * (r[i] - rm[i])) * (inv_deta * inv_deta);
        s0 += (ux * ux + uy * uy + vx * vx + vy * vy) * w_node[j];
    }
};

// power input u F_x (neighbours clamped at the walls): src/diag.cu:350-376
struct PowerInput {
    const double *psi, *a_node, *y, *w_node;
    int Nx, Ny, nforce;
    double inv_deta, h, F0;
    __device__ void operator()(int i, int j, double& s0, double&) const {
        const int ym = j == 0 ? 0 : j - 1, yp = j == Ny - 1 ? Ny - 1 : j + 1;
        const double u = (psi[(size_t)yp * Nx + i] - psi[(size_t)ym * Nx + i]) * 0.5 * inv_deta * a_node[j];
        const double Fx = F0 * sin((double)nforce * kPiD * ((y[j] + h) / (2.0 * h)));
        s0 += u * Fx * w_node[j];
    }
};

// enstrophy input omega f_omega, all rows (full) or interior rows: src/diag.cu:378-466
struct EnstInput {
    const double *w, *y, *w_node;
    int Nx, Ny, nforce, interior;
    double h, F0;
    __device__ void operator()(int i, int j, double& s0, double&) const {
        if (interior && (j == 0 || j == Ny - 1)) return;
        s0 += w[(size_t)j * Nx + i] * f_omega(y[j], h, F0, nforce) * w_node[j];
    }
};

// Omega and omega lap(omega) on the interior rows, the Laplacian in the stencil of the rhs:
// src/diag.cu:103-153, 593-626
struct EnstDissBalance {
    const double *w, *a_node, *a_edge, *w_node;
    int Nx, Ny;
    double inv_dx2, inv_deta2;
    __device__ void operator()(int i, int j, double& s0, double& s1) const {
        if (j == 0 || j == Ny - 1) return;
        const size_t c = (size_t)j * Nx + i;
        const double* r = w + (size_t)j * Nx;
        const double dxx = (r[wrap_x(i + 1, Nx)] - 2 * r[i] + r[wrap_x(i - 1, Nx)]) * inv_dx2;
        const double dyy = a_node[j] * (a_edge[j] * (w[c + Nx] - w[c]) - a_edge[j - 1] * (w[c] - w[c - Nx])) * inv_deta2;
        const double wc = w[c], wt = w_node[j];
        s0 += wt * (wc * wc);
        s1 += wt * (wc * (dxx + dyy));
    }
};

// <omega rhs> over all rows: src/diag.cu:628-691
struct OmegaRhs {
    const double *w, *rhs, *w_node;
    int Nx;
    __device__ void operator()(int i, int j, double& s0, double&) const {
        const size_t c = (size_t)j * Nx + i;
        s0 += w_node[j] * w[c] * rhs[c];
    }
};

// row sums of u, v, u^2, v^2, u v (neighbours clamped at the walls), one CTA per row: src/diag.cu:468-499
__global__ void __launch_bounds__(kRedThreads) k_row_moments(const double* __restrict__ psi, int Nx, int Ny,
                                                             double inv_dx, double inv_deta,
                                                             const double* __restrict__ a_node, double* su,
                                                             double* sv, double* su2, double* sv2, double* suv) {
    const int j = blockIdx.x;
    const int ym = j == 0 ? 0 : j - 1, yp = j == Ny - 1 ? Ny - 1 : j + 1;
    double m[5] = {0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < Nx; i += blockDim.x) {
        const double u = (psi[(size_t)yp * Nx + i] - psi[(size_t)ym * Nx + i]) * 0.5 * inv_deta * a_node[j];
        const double* r = psi + (size_t)j * Nx;
        const double v = -(r[wrap_x(i + 1, Nx)] - r[wrap_x(i - 1, Nx)]) * 0.5 * inv_dx;
        m[0] += u; m[1] += v; m[2] += u * u; m[3] += v * v; m[4] += u * v;
    }
    __shared__ double sh[5][kRedThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < 5; ++q) {
        for (int o = 16; o > 0; o >>= 1) m[q] += __shfl_down_sync(0xffffffffu, m[q], o);
        if (lane == 0) sh[q][warp] = m[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double* out[5] = {su, sv, su2, sv2, suv};
        for (int q = 0; q < 5; ++q) {
            double t = 0.0;
            for (int w = 0; w < kRedThreads / 32; ++w) t += sh[q][w];
            out[q][j] = t;
        }
    }
}

// x-means of the wall rows of omega (with_flux = 0), or of omega omega_y with second-order
// one-sided eta differences (with_flux = 1); one CTA: src/diag.cu:500-583
__global__ void __launch_bounds__(kRedThreads) k_wall_means(const double* __restrict__ w, int Nx, int Ny,
                                                            double inv_deta, const double* __restrict__ a_node,
                                                            int with_flux, double* mb, double* mt) {
    double lb = 0.0, lt = 0.0;
    const double* top = w + (size_t)(Ny - 1) * Nx;
    for (int i = threadIdx.x; i < Nx; i += blockDim.x) {
        if (!with_flux) {
            lb += w[i];
            lt += top[i];
        } else {
            const double w0 = w[i], w1 = w[i + Nx], w2 = w[i + 2 * (size_t)Nx];
            lb += w0 * (a_node[0] * ((-3.0 * w0 + 4.0 * w1 - 1.0 * w2) * (0.5 * inv_deta)));
            const double wN = top[i], wN1 = top[i - Nx], wN2 = top[i - 2 * (size_t)Nx];
            lt += wN * (a_node[Ny - 1] * ((3.0 * wN - 4.0 * wN1 + 1.0 * wN2) * (0.5 * inv_deta)));
        }
    }
    __shared__ double sb[kRedThreads / 32], st[kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        lb += __shfl_down_sync(0xffffffffu, lb, o);
        lt += __shfl_down_sync(0xffffffffu, lt, o);
    }
    if ((threadIdx.x & 31) == 0) { sb[threadIdx.x >> 5] = lb; st[threadIdx.x >> 5] = lt; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0, t = 0.0;
        for (int q = 0; q < kRedThreads / 32; ++q) { b += sb[q]; t += st[q]; }
        *mb = b / (double)Nx;
        *mt = t / (double)Nx;
    }
}

// max |u|, |v|, |v| a over the interior rows (src/diag.cu:702-866), combined in the caller's
// zeroed outputs by atomic maxima on their bit patterns (non-negative doubles order as those)
__global__ void __launch_bounds__(kRedThreads) k_max_uv(const double* __restrict__ psi, int Nx, int Ny, double inv_dx,
                                                        double inv_deta, const double* __restrict__ a_node,
                                                        double* um, double* vm, double* vmm) {
    const size_t N = (size_t)Nx * Ny;
    double mu = 0.0, mv = 0.0, mvm = 0.0;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / (size_t)Nx), i = (int)(idx - (size_t)j * Nx);
        if (j == 0 || j == Ny - 1) continue;
        const double* r = psi + (size_t)j * Nx;
        const double a = a_node[j];
        const double au = fabs(a * ((r[i + Nx] - r[i - Nx]) * (0.5 * inv_deta)));
        const double av = fabs(-((r[wrap_x(i + 1, Nx)] - r[wrap_x(i - 1, Nx)]) * (0.5 * inv_dx)));
        const double avm = av * a;
        if (au > mu) mu = au;
        if (av > mv) mv = av;
        if (avm > mvm) mvm = avm;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mu = fmax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = fmax(mv, __shfl_down_sync(0xffffffffu, mv, o));
        mvm = fmax(mvm, __shfl_down_sync(0xffffffffu, mvm, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(reinterpret_cast<unsigned long long*>(um), (unsigned long long)__double_as_longlong(mu));
        atomicMax(reinterpret_cast<unsigned long long*>(vm), (unsigned long long)__double_as_longlong(mv));
        atomicMax(reinterpret_cast<unsigned long long*>(vmm), (unsigned long long)__double_as_longlong(mvm));
    }
}

inline dim3 tiles(int Nx, int Ny, dim3 tb) { return dim3((Nx + tb.x - 1) / tb.x, (Ny + tb.y - 1) / tb.y); }
inline int lin_blocks(size_t N) { return (int)std::max<size_t>(1, (N + 255) / 256); }

Config grid_config(const Grid& G, const Params& P) {
    Config c;
    c.Nx = G.Nx; c.Ny = G.Ny; c.Lx = G.Lx; c.h = G.h;
    c.beta = P.beta;
    if (P.stretch == "none" || P.stretch == "uniform") c.stretch = 0;
    else if (P.stretch == "tanh") c.stretch = 1;
    else if (P.stretch == "table") {
        if (P.ytable.empty() || P.ytable == "none") throw std::runtime_error("--ytable required for --stretch table");
        std::string err;
        if (!nse2d_host::read_y_table(P.ytable, G.Ny, c.y_table, err)) throw std::runtime_error("--ytable: " + err);
        c.stretch = 2;
    } else {
        throw std::runtime_error("Unknown --stretch '" + P.stretch + "'");
    }
    return c;
}

}  // namespace
}  // namespace nse2d

using namespace nse2d;

// ---- grid metrics (src/grid.cu:7-94) ----
void build_y_metrics(const Grid& Gin, const Params& P, Grid& Gout) {
    const Config c = grid_config(Gin, P);
    Grid g = Gin;
    if (nse2d::build_y_metrics(c, g.y, g.a_node, g.a_edge, g.dy_edge, g.w_node) != 0)
        throw std::runtime_error(nse2d::get_error());
    Gout = g;
}

// ---- src/ops.cuh launchers ----
void launch_uv_from_psi_mapped(const Real* psi, Real* u, Real* v, int Nx, int Ny, Real inv_dx, Real inv_deta,
                               const Real* d_a_node, cudaStream_t s) {
    testapi_uv_from_psi_mapped(psi, u, v, Nx, Ny, inv_dx, inv_deta, d_a_node, s);
}
void launch_omega_from_psi_interior_mapped(Real* w, const Real* psi, int Nx, int Ny, Real inv_dx2, Real inv_deta2,
                                           const Real* d_a_node, const Real* d_a_edge, cudaStream_t s) {
    testapi_omega_from_psi_interior_mapped(w, psi, Nx, Ny, inv_dx2, inv_deta2, d_a_node, d_a_edge, s);
}
void launch_thom_wall_vorticity_mapped(Real* w, const Real* psi, int Nx, int Ny, const Real* d_dy_edge, Real psi_bot,
                                       Real psi_top, cudaStream_t s) {
    testapi_thom_wall_vorticity_mapped(w, psi, Nx, Ny, d_dy_edge, psi_bot, psi_top, s);
}
void launch_arakawa_J_mapped(const Real* psi, const Real* omg, Real* J, int Nx, int Ny, Real inv_dx, Real inv_deta,
                             const Real* d_a_node, cudaStream_t s) {
    testapi_arakawa_J_mapped(psi, omg, J, Nx, Ny, inv_dx, inv_deta, d_a_node, s);
}
void launch_laplacian_fd_mapped(const Real* d_q, Real* d_out, int Nx, int Ny, Real inv_dx2, Real inv_deta2,
                                const Real* d_a_node, const Real* d_a_edge, cudaStream_t s) {
    const dim3 tb(32, 4);
    k_laplacian<<<tiles(Nx, Ny, tb), tb, 0, s>>>(d_q, d_out, Nx, Ny, inv_dx2, inv_deta2, d_a_node, d_a_edge);
    compat_check_launch("launch_laplacian_fd_mapped");
}
void launch_rhs_mapped(const Real* J, const Real* lap, const Real* omg, Real* rhs, int Nx, int Ny, Real nu, Real F0,
                       int nforce, Real h, Real lin_drag, const Real* d_y_node, cudaStream_t s) {
    const dim3 tb(32, 8);
    k_rhs<<<tiles(Nx, Ny, tb), tb, 0, s>>>(J, lap, omg, rhs, Nx, Ny, nu, F0, nforce, h, lin_drag, d_y_node);
    compat_check_launch("launch_rhs_mapped");
}
void launch_mms_add_forcing(Real* d_rhs, int Nx, int Ny, Real Lx, Real h, Real t, Real nu, Real r, Real A0, Real eps,
                            Real Om, int kx_mode, const Real* d_y_node, cudaStream_t s) {
    const size_t N = (size_t)Nx * Ny;
    k_mms_add<<<(int)std::min<size_t>(8192, (N + 255) / 256), 256, 0, s>>>(d_rhs, Nx, Ny, Lx, h, t, nu, r, A0, eps,
                                                                         Om, kx_mode, d_y_node);
    compat_check_launch("launch_mms_add_forcing");
}
void launch_axpy(Real* y, const Real* x, const Real* r, Real dt, size_t N, cudaStream_t s) {
    k_axpy<<<lin_blocks(N), 256, 0, s>>>(y, x, r, dt, N);
    compat_check_launch("launch_axpy");
}
void launch_ssprk2(Real* w2, const Real* w, const Real* w1, const Real* rhs, Real dt, size_t N, cudaStream_t s) {
    k_ssprk2<<<lin_blocks(N), 256, 0, s>>>(w2, w, w1, rhs, dt, N);
    compat_check_launch("launch_ssprk2");
}
void launch_ssprk3(Real* wnp1, const Real* w, const Real* w2, const Real* rhs, Real dt, size_t N, cudaStream_t s) {
    k_ssprk3<<<lin_blocks(N), 256, 0, s>>>(wnp1, w, w2, rhs, dt, N);
    compat_check_launch("launch_ssprk3");
}

// ---- src/diag.cuh launchers ----
void launch_enstrophy_diss_mapped(const Real* omg, int Nx, int Ny, Real inv_dx, Real inv_deta, const Real* d_a_node,
                                  const Real* d_w_node, Real* d_sum_w2, Real* d_sum_gw2, cudaStream_t s) {
    sum2("launch_enstrophy_diss_mapped", EnstDiss{omg, d_a_node, d_w_node, Nx, inv_dx, inv_deta, Ny}, Nx, Ny,
         d_sum_w2, d_sum_gw2, s);
}
void launch_enstrophy_diss_mapped_full(const Real* omg, int Nx, int Ny, Real inv_dx, Real inv_deta,
                                       const Real* d_a_node, const Real* d_w_node, Real* d_sum_w2_full,
                                       Real* d_sum_gw2_full, cudaStream_t s) {
    sum2("launch_enstrophy_diss_mapped_full", EnstDissFull{omg, d_a_node, d_w_node, Nx, Ny, inv_dx, inv_deta}, Nx, Ny,
         d_sum_w2_full, d_sum_gw2_full, s);
}
void launch_enstrophy_sbp_mapped(const Real* omg, int Nx, int Ny, Real inv_dx, Real inv_deta, const Real* d_a_edge,
                                 const Real* d_wt_node, Real* d_sum_eta_h, Real* d_sum_phi_h, cudaStream_t s) {
    sum2("launch_enstrophy_sbp_mapped", EnstSbp{omg, d_a_edge, d_wt_node, Nx, Ny, inv_dx, inv_deta}, Nx, Ny,
         d_sum_eta_h, d_sum_phi_h, s);
}
void launch_kinetic_energy_mapped(const Real* psi, int Nx, int Ny, Real inv_dx, Real inv_deta, const Real* d_a_node,
                                  const Real* d_w_node, Real* d_sum, cudaStream_t s) {
    sum2("launch_kinetic_energy_mapped", KineticEnergy{psi, d_a_node, d_w_node, Nx, Ny, inv_dx, inv_deta}, Nx, Ny,
         d_sum, nullptr, s);
}
void launch_energy_dissipation_mapped(const Real* d_psi, const Real* d_omega, int Nx, int Ny, Real inv_dx,
                                      Real inv_deta, const Real* d_a_node, const Real* d_a_edge, const Real* d_w_node,
                                      Real* d_sum_eps, cudaStream_t s) {
    sum2("launch_energy_dissipation_mapped",
         EnergyDiss{d_psi, d_omega, d_a_node, d_a_edge, d_w_node, Nx, Ny, inv_dx, inv_deta}, Nx, Ny, d_sum_eps,
         nullptr, s);
}
void launch_power_input_mapped(const Real* psi, int Nx, int Ny, Real inv_deta, Real h, Real F0, int nforce,
                               const Real* d_a_node, const Real* d_y_node, const Real* d_w_node, Real* d_sum,
                               cudaStream_t s) {
    sum2("launch_power_input_mapped", PowerInput{psi, d_a_node, d_y_node, d_w_node, Nx, Ny, nforce, inv_deta, h, F0},
         Nx, Ny, d_sum, nullptr, s);
}
void launch_enstrophy_input_mapped_full(const Real* omega, int Nx, int Ny, Real h, Real F0, int nforce,
                                        const Real* d_y_node, const Real* d_w_node, Real* d_sum, cudaStream_t s) {
    sum2("launch_enstrophy_input_mapped_full", EnstInput{omega, d_y_node, d_w_node, Nx, Ny, nforce, 0, h, F0}, Nx,
         Ny, d_sum, nullptr, s);
}
void launch_enstrophy_input_mapped(const Real* omega, int Nx, int Ny, Real h, Real F0, int nforce,
                                   const Real* d_y_node, const Real* d_w_node, Real* d_sum, cudaStream_t s) {
    sum2("launch_enstrophy_input_mapped", EnstInput{omega, d_y_node, d_w_node, Nx, Ny, nforce, 1, h, F0}, Nx, Ny,
         d_sum, nullptr, s);
}
void launch_row_moments_from_psi_mapped(const Real* psi, int Nx, int Ny, Real inv_dx, Real inv_deta,
                                        const Real* d_a_node, Real* su, Real* sv, Real* su2, Real* sv2, Real* suv,
                                        cudaStream_t s) {
    k_row_moments<<<Ny, kRedThreads, 0, s>>>(psi, Nx, Ny, inv_dx, inv_deta, d_a_node, su, sv, su2, sv2, suv);
    compat_check_launch("launch_row_moments_from_psi_mapped");
}
void launch_mean_wall_omega(const Real* omega, int Nx, int Ny, Real* d_mean_bot, Real* d_mean_top, cudaStream_t s) {
    k_wall_means<<<1, kRedThreads, 0, s>>>(omega, Nx, Ny, 0.0, nullptr, 0, d_mean_bot, d_mean_top);
    compat_check_launch("launch_mean_wall_omega");
}
void launch_mean_wall_omega_omegay_mapped(const Real* omega, int Nx, int Ny, Real inv_deta, const Real* d_a_node,
                                          Real* d_mean_bot, Real* d_mean_top, cudaStream_t s) {
    k_wall_means<<<1, kRedThreads, 0, s>>>(omega, Nx, Ny, inv_deta, d_a_node, 1, d_mean_bot, d_mean_top);
    compat_check_launch("launch_mean_wall_omega_omegay_mapped");
}
void launch_enstrophy_diss_balance_mapped(const Real* d_omega, int Nx, int Ny, Real inv_dx2, Real inv_deta2,
                                          const Real* d_a_node, const Real* d_a_edge, const Real* d_w_node,
                                          Real* d_sum_w2, Real* d_sum_eta, cudaStream_t s) {
    sum2("launch_enstrophy_diss_balance_mapped",
         EnstDissBalance{d_omega, d_a_node, d_a_edge, d_w_node, Nx, Ny, inv_dx2, inv_deta2}, Nx, Ny, d_sum_w2,
         d_sum_eta, s);
}
void launch_omega_rhs_balance_mapped(const Real* d_omega, const Real* d_rhs, int Nx, int Ny, const Real* d_w_node,
                                     Real* d_sum_omega_rhs, cudaStream_t stream) {
    sum2("launch_omega_rhs_balance_mapped", OmegaRhs{d_omega, d_rhs, d_w_node, Nx}, Nx, Ny, d_sum_omega_rhs, nullptr,
         stream);
}
void launch_max_uv_from_psi_mapped(const Real* d_psi, int Nx, int Ny, Real inv_dx, Real inv_deta,
                                   const Real* d_a_node, Real* d_umax, Real* d_vmax, Real* d_vmaxm,
                                   cudaStream_t stream) {
    cudaMemsetAsync(d_umax, 0, sizeof(Real), stream);
    cudaMemsetAsync(d_vmax, 0, sizeof(Real), stream);
    cudaMemsetAsync(d_vmaxm, 0, sizeof(Real), stream);
    if (Nx < 2 || Ny < 3) return;
    const size_t N = (size_t)Nx * Ny;
    k_max_uv<<<(int)std::min<size_t>(4096, (N + kRedThreads - 1) / kRedThreads), kRedThreads, 0, stream>>>(
        d_psi, Nx, Ny, inv_dx, inv_deta, d_a_node, d_umax, d_vmax, d_vmaxm);
    compat_check_launch("launch_max_uv_from_psi_mapped");
}

// ---- Spectra1D: a solver context of the grid provides the row transform and the accumulator ----
void Spectra1D::init(const Grid& G) {
    if (impl) context_destroy(static_cast<Context*>(impl));
    Config c;
    c.Nx = G.Nx; c.Ny = G.Ny; c.Lx = G.Lx; c.h = G.h;
    Context* ctx = nullptr;
    if (context_create(c, &ctx) != 0) throw std::runtime_error(std::string("Spectra1D: ") + get_error());
    impl = ctx;
    Nx = G.Nx; Ny = G.Ny; Nxc = Nx / 2 + 1;
    samples = 0;
}
void Spectra1D::accumulate(Real* d_u, Real* d_v) {
    Context* c = static_cast<Context*>(impl);
    if (!c || spectra_accumulate_uv(c, d_u, d_v, 0) != 0) {
        std::fprintf(stderr, "Spectra1D::accumulate: %s\n", c ? get_error() : "not initialised");
        std::abort();
    }
    samples = c->spec_samples;
}
void Spectra1D::write_csv(const std::string& path) {
    Context* c = static_cast<Context*>(impl);
    std::vector<double> acc(2 * (size_t)(c ? c->Hp : 0), 0.0);
    if (c && c->spec_acc) {
        cudaMemcpy(acc.data(), c->spec_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost);
    }
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return;
    std::fprintf(f, "kx,E_u,E_v,E_tot\n");
    for (int k = 0; c && k < Nxc; ++k) {
        const double kx = (2.0 * kPiD * (double)k) / c->cfg.Lx;
        double eu = acc[k], ev = acc[(size_t)c->Hp + k];
        if (samples > 0) { eu /= samples; ev /= samples; }
        std::fprintf(f, "%.10e,%.10e,%.10e,%.10e\n", kx, eu, ev, eu + ev);
    }
    std::fclose(f);
}
Spectra1D::~Spectra1D() {
    if (impl) context_destroy(static_cast<Context*>(impl));
}

// ---- Poisson2D_Z2Z: a solver context whose metrics are the given ones ----
struct Poisson2D_Z2Z::Impl {
    Context* c = nullptr;
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
};

static Context* poisson_context(int Nx, int Ny, double Lx, double h, const std::vector<double>* a_node,
                                const std::vector<double>* a_edge) {
    Config cfg;
    cfg.Nx = Nx; cfg.Ny = Ny; cfg.Lx = Lx; cfg.h = h;
    if (a_node) { cfg.a_node_in = *a_node; cfg.a_edge_in = *a_edge; }
    Context* c = nullptr;
    if (context_create(cfg, &c) != 0) throw std::runtime_error(std::string("Poisson2D_Z2Z: ") + get_error());
    return c;
}

Poisson2D_Z2Z::Poisson2D_Z2Z(const Grid& G, cudaStream_t) : Nx(G.Nx), Ny(G.Ny), Lx_(G.Lx), h_(G.h) {
    impl_ = new Impl();
    impl_->c = poisson_context(Nx, Ny, Lx_, h_, nullptr, nullptr);
    for (auto& ev : impl_->e) cudaEventCreate(&ev);
}

Poisson2D_Z2Z::~Poisson2D_Z2Z() {
    if (!impl_) return;
    if (impl_->c) context_destroy(impl_->c);
    for (auto& ev : impl_->e) if (ev) cudaEventDestroy(ev);
    delete impl_;
}

void Poisson2D_Z2Z::enable_mapped(const Real* a_node, const Real* a_edge, Real inv_deta, cudaStream_t s) {
    mapped = true;
    d_a_node = a_node;
    d_a_edge = a_edge;
    inv_deta2 = inv_deta * inv_deta;
    std::vector<double> an(Ny), ae(Ny - 1);
    cudaMemcpyAsync(an.data(), a_node, Ny * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ae.data(), a_edge, (Ny - 1) * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        std::fprintf(stderr, "Poisson2D_Z2Z::enable_mapped: %s\n", cudaGetErrorString(cudaGetLastError()));
        std::abort();
    }
    context_destroy(impl_->c);
    impl_->c = poisson_context(Nx, Ny, Lx_, h_, &an, &ae);
}

void Poisson2D_Z2Z::solve(const Real* d_omega, Real* d_psi, Real, Real psi_bot, Real psi_top, cudaStream_t s) {
    Context* c = impl_->c;
    c->psi_bot = psi_bot;          // the Dirichlet values of kx = 0 for this solve
    c->psi_top = psi_top;
    cudaEvent_t* e = impl_->e;
    int rc = 0;
    if (profile) cudaEventRecord(e[0], s);
    rc |= launch_fft_fwd(c, d_omega, s);
    if (profile) { cudaEventRecord(e[1], s); cudaEventRecord(e[2], s); }
    rc |= launch_thomas(c, s);
    if (profile) cudaEventRecord(e[3], s);
    if (profile) {
        cudaEventSynchronize(e[3]);
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, e[0], e[1]);
        cudaEventElapsedTime(&b, e[2], e[3]);
        acc_fft_ms += a;
        acc_tridiag_ms += b;
        cudaEventRecord(e[0], s);
    }
    rc |= launch_ifft_thom(c, d_psi, nullptr, 0, false, false, s);
    if (profile) {
        cudaEventRecord(e[1], s);
        cudaEventSynchronize(e[1]);
        float a = 0;
        cudaEventElapsedTime(&a, e[0], e[1]);
        acc_fft_ms += a;
    }
    if (rc != 0) {
        std::fprintf(stderr, "Poisson2D_Z2Z::solve: %s\n", get_error());
        std::abort();
    }
}
