// CPU FP64 oracle for the nse2d channel time step. TEST INFRASTRUCTURE ONLY.
//
// A restatement, written for this project, of the FP64 algorithm of the reference
// (xupingxie/nse2d-channel-gpu). Every function cites the reference file:line it
// follows (paths inside the reference project). Only tests/, the smoke check and
// the CPU baseline / reference arm of bench.py use this library; the CUDA product
// never links it.
//
// Build: oracle/Makefile (g++ -O3 -fopenmp -ffp-contract=off). No FMA contraction is
// allowed, so that results are identical on every x86-64 host.
#include "nse2d_oracle.h"

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;
constexpr double kPi = 3.14159265358979323846264338327950288;   // CUDART_PI / M_PI as a double

// ---------------------------------------------------------------------------------------
// Compensated (Neumaier) sum. The reference accumulates with atomicAdd in arbitrary order
// (src/diag.cu:27,89,...); the oracle uses a deterministic, compensated order instead.
// ---------------------------------------------------------------------------------------
struct KSum {
    double s = 0.0, c = 0.0;
    void add(double x) {
        double t = s + x;
        if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x; else c += (x - t) + s;
        s = t;
    }
    double get() const { return s + c; }
};

// ---------------------------------------------------------------------------------------
// FFT. The reference calls cuFFT Z2Z (src/poisson.cuh:36-37,96,110), a closed library.
// The oracle restates the discrete Fourier transform with its own iterative radix-2
// Cooley-Tukey transform (power-of-two lengths) or a direct O(N^2) sum (other lengths).
// Twiddles exp(-2 pi i k / N) are evaluated in long double and rounded once.
// Forward is unnormalised with e^{-i}; inverse is unnormalised with e^{+i} (cuFFT's
// convention); the reference scales by 1/Nx after the inverse (src/poisson.cuh:114).
// ---------------------------------------------------------------------------------------
struct FFTPlan {
    int n = 0;
    bool pow2 = false;
    std::vector<cplx> tw;      // n entries: exp(-2 pi i k / n)
    std::vector<int> rev;
    explicit FFTPlan(int n_) : n(n_) {
        pow2 = (n > 0) && ((n & (n - 1)) == 0);
        tw.resize(n);
        for (int k = 0; k < n; ++k) {
            long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
            tw[k] = cplx((double)cosl(ang), (double)sinl(ang));
        }
        if (pow2) {
            rev.resize(n);
            int lg = 0; while ((1 << lg) < n) ++lg;
            for (int i = 0; i < n; ++i) {
                int r = 0; for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b);
                rev[i] = r;
            }
        }
    }
    void run(cplx* a, bool inverse, std::vector<cplx>& scratch) const {
        if (!pow2) {                       // direct DFT
            scratch.assign(a, a + n);
            for (int k = 0; k < n; ++k) {
                cplx s(0.0, 0.0);
                for (int m = 0; m < n; ++m) {
                    cplx w = tw[(int)(((int64_t)k * m) % n)];
                    if (inverse) w = std::conj(w);
                    s += scratch[m] * w;
                }
                a[k] = s;
            }
            return;
        }
        for (int i = 0; i < n; ++i) if (i < rev[i]) std::swap(a[i], a[rev[i]]);
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1, step = n / len;
            for (int i = 0; i < n; i += len) {
                for (int j = 0; j < half; ++j) {
                    cplx w = tw[j * step];
                    if (inverse) w = std::conj(w);
                    const cplx u = a[i + j];
                    const cplx v = a[i + j + half] * w;
                    a[i + j] = u + v;
                    a[i + j + half] = u - v;
                }
            }
        }
    }
};

std::shared_ptr<const FFTPlan> get_plan(int n) {
    static std::mutex mu;
    static std::map<int, std::shared_ptr<const FFTPlan>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(n);
    if (it != cache.end()) return it->second;
    auto p = std::make_shared<const FFTPlan>(n);
    cache[n] = p;
    return p;
}

inline int wrapx(int i, int Nx) { return i < 0 ? i + Nx : (i >= Nx ? i - Nx : i); }
inline size_t IX(int j, int i, int Nx) { return (size_t)j * (size_t)Nx + (size_t)i; }

}  // namespace

extern "C" {

void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------------------------------------------------------------------------------
// Grid metrics: src/grid.cu:7-94 (uniform :10-26, tanh :33-45, edges/weights :83-93).
// ---------------------------------------------------------------------------------------
int or_grid_metrics(int Nx, int Ny, double Lx, double h, int stretch, double beta,
                    double* y, double* a_node, double* a_edge, double* dy_edge, double* w_node) {
    (void)Nx; (void)Lx;
    if (Ny < 2) return -1;
    if (Ny <= 2 || stretch == 0) {
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
    if (stretch != 1) return -2;
    const double b = (beta > 0 ? beta : 2.5);
    for (int j = 0; j < Ny; ++j) {
        const double e = -1.0 + 2.0 * (double)j / (double)(Ny - 1);
        y[j] = h * std::tanh(b * e) / std::tanh(b);
    }
    for (int j = 0; j < Ny; ++j) {
        const double e = -1.0 + 2.0 * (double)j / (double)(Ny - 1);
        const double sech = 1.0 / std::cosh(b * e);
        const double y_eta = h * b * (sech * sech) / std::tanh(b);
        a_node[j] = 1.0 / y_eta;
    }
    for (int j = 0; j < Ny - 1; ++j) a_edge[j] = 0.5 * (a_node[j] + a_node[j + 1]);
    for (int j = 0; j < Ny - 1; ++j) dy_edge[j] = y[j + 1] - y[j];
    for (int j = 0; j < Ny; ++j) w_node[j] = 0.0;
    w_node[0] = 0.5 * dy_edge[0];
    w_node[Ny - 1] = 0.5 * dy_edge[Ny - 2];
    for (int j = 1; j < Ny - 1; ++j) w_node[j] = 0.5 * (dy_edge[j - 1] + dy_edge[j]);
    return 0;
}

// ---------------------------------------------------------------------------------------
// Operators: src/ops.cu
// ---------------------------------------------------------------------------------------
// u = a psi_eta / (2 deta), v = -psi_x, clamped j+-1 at the walls: ops.cu:47-63
void or_uv_from_psi(const double* psi, double* u, double* v, int Nx, int Ny,
                    double inv_dx, double inv_deta, const double* a_node) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        const int ym = (iy == 0 ? 0 : iy - 1), yp = (iy == Ny - 1 ? Ny - 1 : iy + 1);
        for (int ix = 0; ix < Nx; ++ix) {
            const int xm = wrapx(ix - 1, Nx), xp = wrapx(ix + 1, Nx);
            const double dpsideta = (psi[IX(yp, ix, Nx)] - psi[IX(ym, ix, Nx)]) * 0.5 * inv_deta;
            const double dpsidx = (psi[IX(iy, xp, Nx)] - psi[IX(iy, xm, Nx)]) * 0.5 * inv_dx;
            u[IX(iy, ix, Nx)] = a_node[iy] * dpsideta;
            v[IX(iy, ix, Nx)] = -dpsidx;
        }
    }
}

// omega = -(dxx psi + mapped dyy psi) on interior rows: ops.cu:72-93
void or_omega_from_psi_interior(double* w, const double* psi, int Nx, int Ny,
                                double inv_dx2, double inv_deta2,
                                const double* a_node, const double* a_edge) {
#pragma omp parallel for schedule(static)
    for (int iy = 1; iy < Ny - 1; ++iy) {
        for (int ix = 0; ix < Nx; ++ix) {
            const int xm = wrapx(ix - 1, Nx), xp = wrapx(ix + 1, Nx);
            const size_t c = IX(iy, ix, Nx);
            const double lapx = psi[IX(iy, xp, Nx)] - 2.0 * psi[c] + psi[IX(iy, xm, Nx)];
            const double aN = a_node[iy], ap = a_edge[iy], am = a_edge[iy - 1];
            const double lapy = aN * (ap * (psi[IX(iy + 1, ix, Nx)] - psi[c]) - am * (psi[c] - psi[IX(iy - 1, ix, Nx)]));
            w[c] = -(inv_dx2 * lapx + inv_deta2 * lapy);
        }
    }
}

// Thom wall vorticity, second order on the stretched grid: ops.cu:102-158
void or_thom(double* w, const double* psi, int Nx, int Ny, const double* dy_edge,
             double psi_bot, double psi_top, int free_slip) {
    if (free_slip) {
        for (int i = 0; i < Nx; ++i) { w[i] = 0; w[IX(Ny - 1, i, Nx)] = 0; }
        return;
    }
    {
        const double dy1 = dy_edge[0], dy2 = dy_edge[1];
        const double A = 2.0 * (1.0 / (dy1 * dy1) + 1.0 / (dy1 * dy2));
        const double B = (-2.0) * dy1 / (dy2 * (dy1 + dy2) * (dy1 + dy2));
        for (int i = 0; i < Nx; ++i) {
            const double d1 = psi[IX(1, i, Nx)] - psi_bot, d2 = psi[IX(2, i, Nx)] - psi_bot;
            w[i] = -(A * d1 + B * d2);
        }
    }
    {
        const double dy1 = dy_edge[Ny - 2], dy2 = dy_edge[Ny - 3];
        const double A = 2.0 * (1.0 / (dy1 * dy1) + 1.0 / (dy1 * dy2));
        const double B = (-2.0) * dy1 / (dy2 * (dy1 + dy2) * (dy1 + dy2));
        for (int i = 0; i < Nx; ++i) {
            const double d1 = psi[IX(Ny - 2, i, Nx)] - psi_top, d2 = psi[IX(Ny - 3, i, Nx)] - psi_top;
            w[IX(Ny - 1, i, Nx)] = -(A * d1 + B * d2);
        }
    }
}

// Mapped 9-point Arakawa Jacobian, returns u.grad(omega) = -(J1+J2+J3)/3: ops.cu:283-326
static inline void arakawa_point(const double* psi, const double* omg, int Nx, int iy, int ix,
                                 double inv_dx, double inv_deta, double a,
                                 double& J1, double& J2, double& J3) {
    const int xm = wrapx(ix - 1, Nx), xp = wrapx(ix + 1, Nx), ym = iy - 1, yp = iy + 1;
    const size_t cxp = IX(iy, xp, Nx), cxm = IX(iy, xm, Nx);
    const size_t cyp = IX(yp, ix, Nx), cym = IX(ym, ix, Nx);
    const size_t ip_jp = IX(yp, xp, Nx), ip_jm = IX(ym, xp, Nx);
    const size_t im_jp = IX(yp, xm, Nx), im_jm = IX(ym, xm, Nx);
    const double inv4dxde = 0.25 * inv_dx * inv_deta;
    J1 = ((psi[cxp] - psi[cxm]) * (a * (omg[cyp] - omg[cym]))
          - (a * (psi[cyp] - psi[cym])) * (omg[cxp] - omg[cxm])) * inv4dxde;
    J2 = (psi[cxp] * (a * (omg[ip_jp] - omg[ip_jm]))
          - psi[cxm] * (a * (omg[im_jp] - omg[im_jm]))
          - a * (psi[cyp] * (omg[ip_jp] - omg[im_jp])
                 - psi[cym] * (omg[ip_jm] - omg[im_jm]))) * inv4dxde;
    J3 = (-omg[cxp] * (a * (psi[ip_jp] - psi[ip_jm]))
          + omg[cxm] * (a * (psi[im_jp] - psi[im_jm]))
          + a * (omg[cyp] * (psi[ip_jp] - psi[im_jp])
                 - omg[cym] * (psi[ip_jm] - psi[im_jm]))) * inv4dxde;
}

void or_arakawa(const double* psi, const double* w, double* J, int Nx, int Ny,
                double inv_dx, double inv_deta, const double* a_node) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        for (int ix = 0; ix < Nx; ++ix) {
            const size_t c = IX(iy, ix, Nx);
            if (iy == 0 || iy == Ny - 1) { J[c] = 0.0; continue; }
            double J1, J2, J3;
            arakawa_point(psi, w, Nx, iy, ix, inv_dx, inv_deta, a_node[iy], J1, J2, J3);
            const double Jbr = (J1 + J2 + J3) * (1.0 / 3.0);
            J[c] = -Jbr;
        }
    }
}

// split Arakawa outputs, any pointer may be NULL: ops.cu:415-467
void or_arakawa_split(const double* psi, const double* w, double* J1o, double* J2o, double* J3o,
                      double* Jadv, int Nx, int Ny, double inv_dx, double inv_deta,
                      const double* a_node) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        for (int ix = 0; ix < Nx; ++ix) {
            const size_t c = IX(iy, ix, Nx);
            if (iy == 0 || iy == Ny - 1) {
                if (J1o) J1o[c] = 0; if (J2o) J2o[c] = 0; if (J3o) J3o[c] = 0; if (Jadv) Jadv[c] = 0;
                continue;
            }
            double J1, J2, J3;
            arakawa_point(psi, w, Nx, iy, ix, inv_dx, inv_deta, a_node[iy], J1, J2, J3);
            if (J1o) J1o[c] = J1; if (J2o) J2o[c] = J2; if (J3o) J3o[c] = J3;
            if (Jadv) Jadv[c] = -((J1 + J2 + J3) * (1.0 / 3.0));
        }
    }
}

// advective reference u.grad(omega) from (u,v): ops.cu:339-371
void or_adv_from_uv(const double* u, const double* v, const double* omg, double* Jadv, int Nx, int Ny,
                    double inv_dx, double inv_deta, const double* a_node) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        for (int ix = 0; ix < Nx; ++ix) {
            const size_t c = IX(iy, ix, Nx);
            if (iy == 0 || iy == Ny - 1) { Jadv[c] = 0; continue; }
            const int xm = wrapx(ix - 1, Nx), xp = wrapx(ix + 1, Nx);
            const double inv2dx = 0.5 * inv_dx, inv2de = 0.5 * inv_deta, a = a_node[iy];
            const double dx_omg = (omg[IX(iy, xp, Nx)] - omg[IX(iy, xm, Nx)]) * inv2dx;
            const double dy_omg = a * (omg[IX(iy + 1, ix, Nx)] - omg[IX(iy - 1, ix, Nx)]) * inv2de;
            Jadv[c] = u[c] * dx_omg + v[c] * dy_omg;
        }
    }
}

// conservative flux form: ops.cu:372-409
void or_adv_flux(const double* u, const double* v, const double* omg, double* Jadv, int Nx, int Ny,
                 double inv_dx, double inv_deta, const double* a_node) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        for (int ix = 0; ix < Nx; ++ix) {
            const size_t c = IX(iy, ix, Nx);
            if (iy == 0 || iy == Ny - 1) { Jadv[c] = 0; continue; }
            const int xm = wrapx(ix - 1, Nx), xp = wrapx(ix + 1, Nx);
            const size_t cxm = IX(iy, xm, Nx), cxp = IX(iy, xp, Nx);
            const size_t cym = IX(iy - 1, ix, Nx), cyp = IX(iy + 1, ix, Nx);
            const double u_ip = (u[cxp] + u[c]) * 0.5, u_im = (u[c] + u[cxm]) * 0.5;
            const double w_ip = (omg[cxp] + omg[c]) * 0.5, w_im = (omg[c] + omg[cxm]) * 0.5;
            const double dFdx = (u_ip * w_ip - u_im * w_im) * inv_dx;
            const double v_jp = (v[cyp] + v[c]) * 0.5, v_jm = (v[c] + v[cym]) * 0.5;
            const double w_jp = (omg[cyp] + omg[c]) * 0.5, w_jm = (omg[c] + omg[cym]) * 0.5;
            const double dFdy = a_node[iy] * ((v_jp * w_jp - v_jm * w_jm) * (0.5 * inv_deta * 2.0));
            Jadv[c] = dFdx + dFdy;
        }
    }
}

// mapped Laplacian, walls = 0: ops.cu:471-499
void or_laplacian(const double* q, double* out, int Nx, int Ny, double inv_dx2, double inv_deta2,
                  const double* a_node, const double* a_edge) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        for (int ix = 0; ix < Nx; ++ix) {
            const size_t id = IX(iy, ix, Nx);
            if (iy == 0 || iy == Ny - 1) { out[id] = 0.0; continue; }
            const int xm = wrapx(ix - 1, Nx), xp = wrapx(ix + 1, Nx);
            const double dxx = (q[IX(iy, xp, Nx)] - 2 * q[id] + q[IX(iy, xm, Nx)]) * inv_dx2;
            const double a = a_node[iy], ap = a_edge[iy], am = a_edge[iy - 1];
            const double dyy = a * (ap * (q[IX(iy + 1, ix, Nx)] - q[id]) - am * (q[id] - q[IX(iy - 1, ix, Nx)])) * inv_deta2;
            out[id] = dxx + dyy;
        }
    }
}

// rhs = -J + nu lap + f(y) - r omega, Kolmogorov vorticity forcing: ops.cu:515-534
void or_rhs(const double* J, const double* lap, const double* w, double* rhs, int Nx, int Ny,
            double nu, double F0, int nforce, double h, double lin_drag, const double* y) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        double f = 0.0;
        if (F0 != 0.0) {
            const double arg = (double)nforce * kPi * ((y[iy] + h) / (2.0 * h));
            f = -F0 * ((double)nforce * kPi / (2.0 * h)) * std::cos(arg);
        }
        for (int ix = 0; ix < Nx; ++ix) {
            const size_t idx = IX(iy, ix, Nx);
            rhs[idx] = -J[idx] + nu * lap[idx] + f - lin_drag * w[idx];
        }
    }
}

// manufactured-solution forcing added to rhs: ops.cu:559-626
void or_mms_add(double* rhs, int Nx, int Ny, double Lx, double h, double t, double nu, double r,
                double A0, double eps, double Om, int kx_mode, const double* y) {
    const double dx = Lx / (double)Nx;
    const double k = 2.0 * kPi * (double)kx_mode / Lx;
    const double c = kPi / (2.0 * h);
    const double A = A0 * (1.0 + eps * std::sin(Om * t));
    const double Aprime = A0 * (eps * Om * std::cos(Om * t));
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j) {
        const double theta = c * (y[j] + h);
        const double two_th = 2.0 * theta;
        const double s_th = std::sin(theta);
        const double s = s_th * s_th;
        const double cos2 = std::cos(two_th), sin2 = std::sin(two_th);
        const double c2 = c * c;
        const double g = (k * k) * s - 2.0 * c2 * cos2;
        const double gpp = 2.0 * c2 * cos2 * ((k * k) + 4.0 * c2);
        const double c3 = c2 * c;
        for (int i = 0; i < Nx; ++i) {
            const double x = (double)i * dx;
            const double sk = std::sin(k * x), s2k = std::sin(2.0 * k * x);
            const double term_lin = Aprime * g + (nu * A) * ((k * k) * g - gpp) + (r * A) * g;
            const double term_adv = -(A * A) * k * c3 * s2k * sin2;
            rhs[IX(j, i, Nx)] += sk * term_lin + term_adv;
        }
    }
}

// SSPRK(3,3) Shu-Osher combines: ops.cu:644-655
void or_axpy(double* out, const double* x, const double* r, double dt, int64_t N) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) out[i] = x[i] + dt * r[i];
}
void or_ssprk2(double* w2, const double* w, const double* w1, const double* r, double dt, int64_t N) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) w2[i] = 0.75 * w[i] + 0.25 * (w1[i] + dt * r[i]);
}
void or_ssprk3(double* wn, const double* w, const double* w2, const double* r, double dt, int64_t N) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) wn[i] = (1.0 / 3.0) * w[i] + (2.0 / 3.0) * (w2[i] + dt * r[i]);
}

// ---------------------------------------------------------------------------------------
// Poisson: spectral kx^2 (poisson.cu:16-22), elimination table cp (poisson.cu:38-68),
// Thomas sweeps (poisson.cu:70-133), FFT pack/scale (poisson.cuh:83-118).
// ---------------------------------------------------------------------------------------
static double kx2_of(int k, int Nx, double Lx) {
    const int kphys_i = (k <= Nx / 2 ? k : k - Nx);
    const double kphys = (2.0 * kPi * (double)kphys_i) / Lx;
    return kphys * kphys;
}

void or_poisson_cp(double* cp, int Nx, int Ny, double Lx, const double* a_node,
                   const double* a_edge, double inv_deta) {
    const double inv_deta2 = inv_deta * inv_deta;
    const int Ni = Ny - 2;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Nx; ++k) {
        const double kx2 = kx2_of(k, Nx, Lx);
        int j = 1;
        double an = a_node[j], ae_p = a_edge[j], ae_m = a_edge[j - 1];
        double a_sub = an * ae_m * inv_deta2, c_sup = an * ae_p * inv_deta2;
        double b = -(a_sub + c_sup) - kx2;
        double cp_prev = c_sup / b;
        cp[(size_t)k * Ni + 0] = cp_prev;
        for (int r = 1; r < Ni; ++r) {
            j = r + 1;
            an = a_node[j]; ae_p = a_edge[j]; ae_m = a_edge[j - 1];
            a_sub = an * ae_m * inv_deta2; c_sup = an * ae_p * inv_deta2;
            b = -(a_sub + c_sup) - kx2;
            const double den = b - a_sub * cp_prev;
            const double cpi = c_sup / den;
            cp[(size_t)k * Ni + r] = cpi;
            cp_prev = cpi;
        }
    }
}

void or_rfft_rows(const double* in, double* out, int Nx, int Ny) {
    auto plan = get_plan(Nx);
    const int H = Nx / 2 + 1;
#pragma omp parallel
    {
        std::vector<cplx> row(Nx), scratch;
#pragma omp for schedule(static)
        for (int j = 0; j < Ny; ++j) {
            for (int i = 0; i < Nx; ++i) row[i] = cplx(in[IX(j, i, Nx)], 0.0);
            plan->run(row.data(), false, scratch);
            for (int k = 0; k < H; ++k) {
                out[2 * ((size_t)j * H + k)] = row[k].real();
                out[2 * ((size_t)j * H + k) + 1] = row[k].imag();
            }
        }
    }
}

namespace {
// the solve itself, with a precomputed cp table (all Nx columns, as the reference)
void poisson_solve_cp(const double* w, double* psi, int Nx, int Ny, double Lx,
                      const double* a_node, const double* a_edge, double inv_deta,
                      double psi_bot, double psi_top, const double* cp, std::vector<cplx>& hat) {
    const double inv_deta2 = inv_deta * inv_deta;
    const int Ni = Ny - 2;
    auto plan = get_plan(Nx);
    hat.resize((size_t)Nx * Ny);
    // pack real -> complex and forward FFT per row (poisson.cu:8-11, poisson.cuh:96)
#pragma omp parallel
    {
        std::vector<cplx> scratch;
#pragma omp for schedule(static)
        for (int j = 0; j < Ny; ++j) {
            cplx* row = &hat[(size_t)j * Nx];
            for (int i = 0; i < Nx; ++i) row[i] = cplx(w[IX(j, i, Nx)], 0.0);
            plan->run(row, false, scratch);
        }
    }
    // Thomas per kx (poisson.cu:70-133). Columns k and Nx-k carry conjugate data and the
    // same kx^2; the oracle solves k = 0..Nx/2 and mirrors the conjugate.
    const int H = Nx / 2 + 1;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < H; ++k) {
        const double kx2 = kx2_of(k, Nx, Lx);
        const double* cpk = cp + (size_t)k * Ni;
        int j = 1;
        double an = a_node[j], ae_p = a_edge[j], ae_m = a_edge[j - 1];
        double a_sub = an * ae_m * inv_deta2, c_sup = an * ae_p * inv_deta2;
        double b = -(a_sub + c_sup) - kx2;
        cplx rhs0 = -hat[(size_t)Nx * j + k];
        double r0x = rhs0.real(), r0y = rhs0.imag();
        if (k == 0) r0x -= a_sub * psi_bot * (double)Nx;
        const double den0 = b;
        double dpx = (r0x - a_sub * 0.0) / den0, dpy = (r0y - a_sub * 0.0) / den0;
        std::vector<cplx> col(Ni);
        col[0] = cplx(dpx, dpy);
        for (int r = 1; r < Ni; ++r) {
            j = r + 1;
            an = a_node[j]; ae_p = a_edge[j]; ae_m = a_edge[j - 1];
            a_sub = an * ae_m * inv_deta2; c_sup = an * ae_p * inv_deta2;
            const cplx h_ = hat[(size_t)Nx * j + k];
            double rx = -h_.real(), ry = -h_.imag();
            if (k == 0 && r == Ni - 1) rx -= c_sup * psi_top * (double)Nx;
            const double cpj = cpk[r];
            const double den = c_sup / cpj;
            dpx = (rx - a_sub * dpx) / den;
            dpy = (ry - a_sub * dpy) / den;
            col[r] = cplx(dpx, dpy);
        }
        cplx xnext = col[Ni - 1];
        for (int r = Ni - 2; r >= 0; --r) {
            const double cpj = cpk[r];
            const cplx d = col[r];
            const cplx xj(d.real() - cpj * xnext.real(), d.imag() - cpj * xnext.imag());
            col[r] = xj;
            xnext = xj;
        }
        for (int r = 0; r < Ni; ++r) hat[(size_t)Nx * (r + 1) + k] = col[r];
        hat[k] = (k == 0 ? cplx((double)Nx * psi_bot, 0.0) : cplx(0.0, 0.0));
        hat[(size_t)Nx * (Ny - 1) + k] = (k == 0 ? cplx((double)Nx * psi_top, 0.0) : cplx(0.0, 0.0));
    }
    for (int j = 0; j < Ny; ++j)
        for (int k = H; k < Nx; ++k) hat[(size_t)j * Nx + k] = std::conj(hat[(size_t)j * Nx + (Nx - k)]);
    // inverse FFT and scale by 1/Nx (poisson.cu:12-15, poisson.cuh:110-114)
    const double s = 1.0 / (double)Nx;
#pragma omp parallel
    {
        std::vector<cplx> scratch;
#pragma omp for schedule(static)
        for (int j = 0; j < Ny; ++j) {
            cplx* row = &hat[(size_t)j * Nx];
            plan->run(row, true, scratch);
            for (int i = 0; i < Nx; ++i) psi[IX(j, i, Nx)] = s * row[i].real();
        }
    }
}
}  // namespace

void or_poisson_solve(const double* w, double* psi, int Nx, int Ny, double Lx,
                      const double* a_node, const double* a_edge, double inv_deta,
                      double psi_bot, double psi_top) {
    std::vector<double> cp((size_t)Nx * (Ny - 2));
    or_poisson_cp(cp.data(), Nx, Ny, Lx, a_node, a_edge, inv_deta);
    std::vector<cplx> hat;
    poisson_solve_cp(w, psi, Nx, Ny, Lx, a_node, a_edge, inv_deta, psi_bot, psi_top, cp.data(), hat);
}

// ---------------------------------------------------------------------------------------
// Reductions: src/diag.cu
// ---------------------------------------------------------------------------------------
// max |u|, |v|, |v| a over interior rows: diag.cu:702-866
void or_max_uv(const double* psi, int Nx, int Ny, double inv_dx, double inv_deta,
               const double* a_node, double out3[3]) {
    out3[0] = out3[1] = out3[2] = 0.0;
    if (Nx < 2 || Ny < 3) return;
    std::vector<double> ru(Ny, 0.0), rv(Ny, 0.0), rvm(Ny, 0.0);
#pragma omp parallel for schedule(static)
    for (int j = 1; j < Ny - 1; ++j) {
        double um = 0, vm = 0, vmm = 0;
        const double a = a_node[j];
        for (int i = 0; i < Nx; ++i) {
            const int ip = (i + 1 < Nx) ? i + 1 : 0, im = (i > 0) ? i - 1 : Nx - 1;
            const double dpsideta = (psi[IX(j + 1, i, Nx)] - psi[IX(j - 1, i, Nx)]) * (0.5 * inv_deta);
            const double dpsidx = (psi[IX(j, ip, Nx)] - psi[IX(j, im, Nx)]) * (0.5 * inv_dx);
            const double u = a * dpsideta, v = -dpsidx;
            const double au = std::fabs(u), av = std::fabs(v), avm = av * a;
            if (au > um) um = au;
            if (av > vm) vm = av;
            if (avm > vmm) vmm = avm;
        }
        ru[j] = um; rv[j] = vm; rvm[j] = vmm;
    }
    for (int j = 1; j < Ny - 1; ++j) {
        if (ru[j] > out3[0]) out3[0] = ru[j];
        if (rv[j] > out3[1]) out3[1] = rv[j];
        if (rvm[j] > out3[2]) out3[2] = rvm[j];
    }
}

// Per-row compensated sums, then a compensated sum over rows (deterministic order).
void or_diag_sums(const double* psi, const double* w, const double* rhs, const double* J,
                  int Nx, int Ny, double inv_dx, double inv_deta, double h, double F0, int nforce,
                  const double* a_node, const double* a_edge, const double* y,
                  const double* w_node, double* out) {
    const int NS = OR_NSUM;
    std::vector<double> rows((size_t)Ny * NS, 0.0);
    const double inv_dx2 = inv_dx * inv_dx, inv_deta2 = inv_deta * inv_deta;
    const double deta = 2.0 / (double)(Ny - 1);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j) {
        KSum s[OR_NSUM];
        const double wq = w_node[j];
        const double a = a_node[j];
        const double wt = (j >= 1 && j <= Ny - 2) ? deta / a_node[j] : 0.0;   // main.cu:252-254
        const int ym = (j == 0 ? 0 : j - 1), yp = (j == Ny - 1 ? Ny - 1 : j + 1);
        const double yy = y[j];
        const double argF = (double)nforce * kPi * ((yy + h) / (2.0 * h));
        const double Fx = F0 * std::sin(argF);                                   // diag.cu:359
        const double fom = -F0 * ((double)nforce * kPi / (2.0 * h)) * std::cos(argF);  // diag.cu:392-393
        for (int i = 0; i < Nx; ++i) {
            const int xm = (i == 0 ? Nx - 1 : i - 1), xp = (i == Nx - 1 ? 0 : i + 1);
            const size_t c = IX(j, i, Nx);
            const double wc = w[c];
            // kinetic energy, interior rows: diag.cu:201-223
            if (j != 0 && j != Ny - 1) {
                const double u = (psi[IX(j + 1, i, Nx)] - psi[IX(j - 1, i, Nx)]) * 0.5 * inv_deta * a;
                const double v = -(psi[IX(j, xp, Nx)] - psi[IX(j, xm, Nx)]) * 0.5 * inv_dx;
                s[OR_S_K].add(0.5 * (u * u + v * v) * wq);
            }
            // enstrophy and palinstrophy on all rows, one-sided at walls: diag.cu:43-90
            {
                const double wx = (w[IX(j, xp, Nx)] - w[IX(j, xm, Nx)]) * 0.5 * inv_dx;
                double weta;
                if (j == 0) {
                    weta = (-3.0 * w[IX(0, i, Nx)] + 4.0 * w[IX(1, i, Nx)] - 1.0 * w[IX(2, i, Nx)]) * (0.5 * inv_deta);
                } else if (j == Ny - 1) {
                    weta = (3.0 * w[IX(Ny - 1, i, Nx)] - 4.0 * w[IX(Ny - 2, i, Nx)] + 1.0 * w[IX(Ny - 3, i, Nx)]) * (0.5 * inv_deta);
                } else {
                    weta = (w[IX(j + 1, i, Nx)] - w[IX(j - 1, i, Nx)]) * 0.5 * inv_deta;
                }
                const double wy = a * weta;
                s[OR_S_W2].add(wq * (wc * wc));
                s[OR_S_GW2].add(wq * (wx * wx + wy * wy));
                if (j == 0) s[OR_S_WWY_BOT].add(wc * wy);           // diag.cu:516-569
                if (j == Ny - 1) s[OR_S_WWY_TOP].add(wc * wy);
                if (j == 0) s[OR_S_MOB].add(wc);                     // diag.cu:500-507
                if (j == Ny - 1) s[OR_S_MOT].add(wc);
            }
            // <omega rhs> all rows: diag.cu:628-671
            if (rhs) s[OR_S_WRHS].add(wq * wc * rhs[c]);
            // power input: diag.cu:350-367
            {
                const double u = (psi[IX(yp, i, Nx)] - psi[IX(ym, i, Nx)]) * 0.5 * inv_deta * a;
                s[OR_S_PIN].add(u * Fx * wq);
            }
            // energy dissipation: diag.cu:250-329
            if (j == 0 || j == Ny - 1) {
                const double uy = -wc;
                s[OR_S_EPS].add((uy * uy) * wq);
            } else {
                const double ap = a_edge[j], am = a_edge[j - 1];
                const double psi_x_jp = (psi[IX(j + 1, xp, Nx)] - psi[IX(j + 1, xm, Nx)]) * (0.5 * inv_dx);
                const double psi_x_jm = (psi[IX(j - 1, xp, Nx)] - psi[IX(j - 1, xm, Nx)]) * (0.5 * inv_dx);
                const double ux = a * (psi_x_jp - psi_x_jm) * (0.5 * inv_deta);
                const double vy = -ux;
                const double vx = -(psi[IX(j, xp, Nx)] - 2.0 * psi[c] + psi[IX(j, xm, Nx)]) * inv_dx2;
                const double uy = a * (ap * (psi[IX(j + 1, i, Nx)] - psi[c]) - am * (psi[c] - psi[IX(j - 1, i, Nx)])) * inv_deta2;
                const double g2 = ux * ux + uy * uy + vx * vx + vy * vy;
                s[OR_S_EPS].add(g2 * wq);
            }
            // enstrophy input, all rows: diag.cu:378-409
            s[OR_S_POM].add(wc * fom * wq);
            // ---- closure_diag sums (main.cu:595-611) ----
            if (j != 0 && j != Ny - 1) {
                // enstrophy_diss_mapped (interior, centered): diag.cu:6-28, weights w_node and wt
                const double wx = (w[IX(j, xp, Nx)] - w[IX(j, xm, Nx)]) * 0.5 * inv_dx;
                const double wy = a * (w[IX(j + 1, i, Nx)] - w[IX(j - 1, i, Nx)]) * 0.5 * inv_deta;
                s[OR_S_W2_INT].add(wq * (wc * wc));
                s[OR_S_GW2_INT].add(wq * (wx * wx + wy * wy));
                s[OR_S_T2_W2].add(wt * (wc * wc));
                s[OR_S_T2_G2].add(wt * (wx * wx + wy * wy));
            }
            if (rhs) s[OR_S_T2_D].add(wt * wc * rhs[c]);
            if (J) s[OR_S_T2_J].add(wt * wc * J[c]);
            s[OR_S_T2_P].add(wc * fom * wt);
            // SBP remainders: diag.cu:166-190
            if (j >= 1 && j <= Ny - 2) {
                const double dxw = (w[IX(j, xp, Nx)] - wc) * inv_dx;
                s[OR_S_T2_ETA].add(wt * dxw * dxw);
            }
            if (j <= Ny - 2) {
                const double dw = w[IX(j + 1, i, Nx)] - wc;
                s[OR_S_T2_ETA].add(a_edge[j] * dw * dw * inv_deta);
            }
            if (j == 0) s[OR_S_T2_PHI].add(-(wc * a_edge[0] * (w[IX(1, i, Nx)] - wc) * inv_deta));
            if (j == Ny - 1) s[OR_S_T2_PHI].add(wc * a_edge[Ny - 2] * (wc - w[IX(Ny - 2, i, Nx)]) * inv_deta);
            // wall-row part of <omega rhs> with trapezoid weights (main.cu:290-296)
            if (rhs && (j == 0 || j == Ny - 1)) s[OR_S_WALL_WRHS].add(wq * wc * rhs[c]);
        }
        for (int q = 0; q < NS; ++q) rows[(size_t)j * NS + q] = s[q].get();
    }
    for (int q = 0; q < NS; ++q) {
        KSum t;
        for (int j = 0; j < Ny; ++j) t.add(rows[(size_t)j * NS + q]);
        out[q] = t.get();
    }
}

// per-row sums of u, v, u^2, v^2, uv with clamped j+-1: diag.cu:468-492
void or_row_moments(const double* psi, int Nx, int Ny, double inv_dx, double inv_deta,
                    const double* a_node, double* su, double* sv, double* su2, double* sv2,
                    double* suv) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < Ny; ++iy) {
        KSum a, b, c, d, e;
        const int ym = (iy == 0 ? 0 : iy - 1), yp = (iy == Ny - 1 ? Ny - 1 : iy + 1);
        for (int ix = 0; ix < Nx; ++ix) {
            const int xm = (ix == 0 ? Nx - 1 : ix - 1), xp = (ix == Nx - 1 ? 0 : ix + 1);
            const double u = (psi[IX(yp, ix, Nx)] - psi[IX(ym, ix, Nx)]) * 0.5 * inv_deta * a_node[iy];
            const double v = -(psi[IX(iy, xp, Nx)] - psi[IX(iy, xm, Nx)]) * 0.5 * inv_dx;
            a.add(u); b.add(v); c.add(u * u); d.add(v * v); e.add(u * v);
        }
        su[iy] = a.get(); sv[iy] = b.get(); su2[iy] = c.get(); sv2[iy] = d.get(); suv[iy] = e.get();
    }
}

// ---------------------------------------------------------------------------------------
// Solver: setup (main.cu:43-87, 187-215) and one SSPRK(3,3) step (main.cu:482-538)
// ---------------------------------------------------------------------------------------
struct or_solver {
    or_config c{};
    int Nx = 0, Ny = 0;
    size_t N = 0;
    std::vector<double> y, a_node, a_edge, dy_edge, w_node;
    double dx = 0, dy = 0, inv_dx = 0, inv_dx2 = 0, deta = 0, inv_deta = 0, inv_deta2 = 0;
    double dy_min = 0, inv_dymin2 = 0, Ly_full = 0, invA_full = 0, meanFx_A = 0, nu = 0;
    double psi_bot = 0, psi_top = 0;
    std::vector<double> w, w1, w2, psi, rhs, J, lap, cp;
    std::vector<cplx> hat;
    double Jwall[3] = {0, 0, 0};
};

static void solve(or_solver* s, const double* wsrc) {
    poisson_solve_cp(wsrc, s->psi.data(), s->Nx, s->Ny, s->c.Lx, s->a_node.data(), s->a_edge.data(),
                     s->inv_deta, s->psi_bot, s->psi_top, s->cp.data(), s->hat);
}

static double wall_row_enstrophy(const or_solver* s, const double* f) {   // main.cu:284-289
    const int Nx = s->Nx, Ny = s->Ny;
    const double wq_b = s->w_node[0], wq_t = s->w_node[Ny - 1];
    double acc = 0.0;
    for (int i = 0; i < Nx; ++i) {
        const double b = f[i], t = f[IX(Ny - 1, i, Nx)];
        acc += wq_b * b * b + wq_t * t * t;
    }
    return 0.5 * acc * s->invA_full;
}

static void thom_stage(or_solver* s, double* f, int stage) {
    if (s->c.closure_diag) {
        const double Jb = wall_row_enstrophy(s, f);
        or_thom(f, s->psi.data(), s->Nx, s->Ny, s->dy_edge.data(), s->psi_bot, s->psi_top, s->c.free_slip);
        s->Jwall[stage] += wall_row_enstrophy(s, f) - Jb;
    } else {
        or_thom(f, s->psi.data(), s->Nx, s->Ny, s->dy_edge.data(), s->psi_bot, s->psi_top, s->c.free_slip);
    }
}

static void build_rhs(or_solver* s, const double* wsrc, double tm) {
    const int Nx = s->Nx, Ny = s->Ny;
    or_arakawa(s->psi.data(), wsrc, s->J.data(), Nx, Ny, s->inv_dx, s->inv_deta, s->a_node.data());
    or_laplacian(wsrc, s->lap.data(), Nx, Ny, s->inv_dx2, s->inv_deta2, s->a_node.data(), s->a_edge.data());
    or_rhs(s->J.data(), s->lap.data(), wsrc, s->rhs.data(), Nx, Ny, s->nu, s->c.F0, s->c.nforce, s->c.h,
           s->c.lin_drag, s->y.data());
    if (s->c.mms)
        or_mms_add(s->rhs.data(), Nx, Ny, s->c.Lx, s->c.h, tm, s->nu, s->c.lin_drag, s->c.mms_A0,
                   s->c.mms_eps, s->c.mms_Om, s->c.mms_kx, s->y.data());
}

or_solver* or_create(const or_config* cfg) {
    if (!cfg || cfg->Nx < 2 || cfg->Ny < 4) return nullptr;
    auto* s = new or_solver();
    s->c = *cfg;
    s->Nx = cfg->Nx; s->Ny = cfg->Ny; s->N = (size_t)cfg->Nx * cfg->Ny;
    const int Ny = s->Ny;
    s->y.resize(Ny); s->a_node.resize(Ny); s->a_edge.resize(Ny - 1); s->dy_edge.resize(Ny - 1); s->w_node.resize(Ny);
    if (or_grid_metrics(s->Nx, Ny, cfg->Lx, cfg->h, cfg->stretch, cfg->beta, s->y.data(), s->a_node.data(),
                        s->a_edge.data(), s->dy_edge.data(), s->w_node.data()) != 0) {
        delete s;
        return nullptr;
    }
    s->nu = (cfg->nu_override >= 0 ? cfg->nu_override : (2.0 * cfg->h * cfg->Ub) / cfg->Reb);   // common.cuh:69
    s->dx = cfg->Lx / (double)s->Nx;                                                          // common.cuh:54-55
    s->dy = (2.0 * cfg->h) / (double)(Ny - 1);
    s->inv_dx = 1.0 / s->dx; s->inv_dx2 = s->inv_dx * s->inv_dx;                              // main.cu:49-53
    s->deta = (Ny > 1) ? 2.0 / (double)(Ny - 1) : 1.0;
    s->inv_deta = 1.0 / s->deta; s->inv_deta2 = s->inv_deta * s->inv_deta;
    s->dy_min = std::fabs(s->dy_edge[0]);                                                     // main.cu:56-62
    for (int j = 1; j < Ny - 1; ++j) s->dy_min = std::min(s->dy_min, std::fabs(s->dy_edge[j]));
    s->inv_dymin2 = 1.0 / (s->dy_min * s->dy_min);
    s->Ly_full = 0.0;                                                                         // main.cu:65-71
    for (int j = 0; j < Ny; ++j) s->Ly_full += s->w_node[j];
    s->invA_full = 1.0 / ((double)s->Nx * s->Ly_full);
    s->meanFx_A = 0.0;                                                                        // main.cu:78-87
    if (cfg->F0 != 0.0) {
        for (int j = 0; j < Ny; ++j) {
            const double arg = (double)cfg->nforce * kPi * ((s->y[j] + cfg->h) / (2.0 * cfg->h));
            s->meanFx_A += cfg->F0 * std::sin(arg) * s->w_node[j];
        }
        s->meanFx_A /= s->Ly_full;
    }
    s->psi_bot = 0.0; s->psi_top = 2.0 * cfg->h * cfg->Ub;                                   // main.cu:211
    for (auto* v : {&s->w, &s->w1, &s->w2, &s->psi, &s->rhs, &s->J, &s->lap}) v->assign(s->N, 0.0);
    s->cp.resize((size_t)s->Nx * (Ny - 2));
    or_poisson_cp(s->cp.data(), s->Nx, Ny, cfg->Lx, s->a_node.data(), s->a_edge.data(), s->inv_deta);
    return s;
}

void or_destroy(or_solver* s) { delete s; }
int or_nx(const or_solver* s) { return s->Nx; }
int or_ny(const or_solver* s) { return s->Ny; }
double or_nu(const or_solver* s) { return s->nu; }

const double* or_metric(const or_solver* s, int which) {
    switch (which) {
        case 0: return s->y.data();
        case 1: return s->a_node.data();
        case 2: return s->a_edge.data();
        case 3: return s->dy_edge.data();
        case 4: return s->w_node.data();
        default: return nullptr;
    }
}

void or_set_omega(or_solver* s, const double* w) {
    std::memcpy(s->w.data(), w, s->N * sizeof(double));
    solve(s, s->w.data());                                                                    // main.cu:212-213
    or_thom(s->w.data(), s->psi.data(), s->Nx, s->Ny, s->dy_edge.data(), s->psi_bot, s->psi_top, s->c.free_slip);
    s->Jwall[0] = s->Jwall[1] = s->Jwall[2] = 0.0;
}

void or_get_fields(const or_solver* s, double* w, double* psi) {
    if (w) std::memcpy(w, s->w.data(), s->N * sizeof(double));
    if (psi) std::memcpy(psi, s->psi.data(), s->N * sizeof(double));
}

void or_set_fields(or_solver* s, const double* w, const double* psi) {
    std::memcpy(s->w.data(), w, s->N * sizeof(double));
    std::memcpy(s->psi.data(), psi, s->N * sizeof(double));
}

double or_adapt_dt(or_solver* s, double* umax3) {                                            // main.cu:439-458
    double m[3];
    or_max_uv(s->psi.data(), s->Nx, s->Ny, s->inv_dx, s->inv_deta, s->a_node.data(), m);
    if (umax3) { umax3[0] = m[0]; umax3[1] = m[1]; umax3[2] = m[2]; }
    const double dt_x = (m[0] > 0 ? s->c.cfl * (s->dx / m[0]) : 1e30);
    const double dt_y = (m[2] > 0 ? s->c.cfl * (s->deta / m[2]) : 1e30);
    const double dt_adv = std::fmin(dt_x, dt_y);
    const double dt_vis = (s->nu > 0) ? s->c.cvisc * 0.5 / (s->nu * (s->inv_dx2 + s->inv_dymin2)) : 1e30;
    return std::fmin(s->c.dt_max, std::fmin(dt_adv, dt_vis));
}

void or_step(or_solver* s, double t, double dt) {
    const int64_t N = (int64_t)s->N;
    // stage 1 (main.cu:484-501)
    build_rhs(s, s->w.data(), t);
    or_axpy(s->w1.data(), s->w.data(), s->rhs.data(), dt, N);
    solve(s, s->w1.data());
    thom_stage(s, s->w1.data(), 0);
    // stage 2 (main.cu:504-520)
    build_rhs(s, s->w1.data(), t + dt);
    or_ssprk2(s->w2.data(), s->w.data(), s->w1.data(), s->rhs.data(), dt, N);
    solve(s, s->w2.data());
    thom_stage(s, s->w2.data(), 1);
    // stage 3 (main.cu:523-538), in place
    build_rhs(s, s->w2.data(), t + 0.5 * dt);
    or_ssprk3(s->w.data(), s->w.data(), s->w2.data(), s->rhs.data(), dt, N);
    solve(s, s->w.data());
    thom_stage(s, s->w.data(), 2);
}

double or_jwall(const or_solver* s, int stage) { return s->Jwall[stage]; }

// One diagnostics.csv row, columns 4..32 of main.cu:162-163 (umax .. Phi_h).
// t0_row = 1: the t = 0 row of main.cu:325-421 (rhs rebuilt at the state; closure columns
// nan / 0); otherwise the output-time row of main.cu:566-692, where dOmega_rhs pairs the
// state with the stage-3 right-hand side still held from the last step.
void or_diag_row(or_solver* s, double t, int t0_row, double* out) {
    const int Nx = s->Nx, Ny = s->Ny;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    double m[3];
    or_max_uv(s->psi.data(), Nx, Ny, s->inv_dx, s->inv_deta, s->a_node.data(), m);
    double S[OR_NSUM];
    if (t0_row) build_rhs(s, s->w.data(), t);
    or_diag_sums(s->psi.data(), s->w.data(), s->rhs.data(), nullptr, Nx, Ny, s->inv_dx, s->inv_deta,
                 s->c.h, s->c.F0, s->c.nforce, s->a_node.data(), s->a_edge.data(), s->y.data(),
                 s->w_node.data(), S);
    const double nu = s->nu, iA = s->invA_full, h = s->c.h;
    const double K = S[OR_S_K] * iA;
    const double Omega = 0.5 * S[OR_S_W2] * iA;
    const double eta = nu * S[OR_S_GW2] * iA;
    const double mwb = S[OR_S_WWY_BOT] / (double)Nx, mwt = S[OR_S_WWY_TOP] / (double)Nx;
    const double BOm = (nu > 0.0) ? (nu * (mwt - mwb) / (2.0 * h)) : 0.0;
    const double dOm = S[OR_S_WRHS] * iA;
    const double Pin = S[OR_S_PIN] * iA;
    const double eps = nu * S[OR_S_EPS] * iA;
    const double POm = S[OR_S_POM] * iA;
    const double mOb = S[OR_S_MOB] / (double)Nx, mOt = S[OR_S_MOT] / (double)Nx;
    const double tb = -nu * mOb, tt = -nu * mOt;
    const double ut = std::sqrt(0.5 * (std::fabs(tb) + std::fabs(tt)));
    const double Ub = s->c.Ub;
    const double Cf = (Ub != 0.0) ? 2.0 * (0.5 * (std::fabs(tb) + std::fabs(tt))) / (Ub * Ub) : nan;
    const double Ret = (nu > 0.0) ? ut * h / nu : 0.0;
    const double dpdx = (tt - tb) / (2.0 * h) + s->meanFx_A - s->c.lin_drag * Ub;
    double* o = out;
    o[0] = m[0]; o[1] = m[1]; o[2] = K; o[3] = Omega; o[4] = dOm; o[5] = eta; o[6] = BOm; o[7] = Pin;
    o[8] = eps; o[9] = POm; o[10] = tb; o[11] = tt; o[12] = dpdx; o[13] = ut; o[14] = Cf; o[15] = Ret;
    for (int q = 16; q < 29; ++q) o[q] = nan;
    if (!s->c.closure_diag) return;
    if (t0_row) {
        o[16] = dOm; o[20] = 0.0; o[21] = 0.0; o[22] = 0.0;
        return;
    }
    // same-state rebuild (main.cu:595-611)
    build_rhs(s, s->w.data(), t);
    double C[OR_NSUM];
    or_diag_sums(s->psi.data(), s->w.data(), s->rhs.data(), s->J.data(), Nx, Ny, s->inv_dx, s->inv_deta,
                 h, s->c.F0, s->c.nforce, s->a_node.data(), s->a_edge.data(), s->y.data(),
                 s->w_node.data(), C);
    const double same = C[OR_S_WRHS] * iA;
    o[16] = same;
    o[17] = same - C[OR_S_WALL_WRHS] * iA;
    o[18] = 0.5 * C[OR_S_W2_INT] * iA;
    o[19] = nu * C[OR_S_GW2_INT] * iA;
    o[20] = s->Jwall[0]; o[21] = s->Jwall[1]; o[22] = s->Jwall[2];
    o[23] = 0.5 * C[OR_S_T2_W2] * iA;
    o[24] = C[OR_S_T2_D] * iA;
    o[25] = -C[OR_S_T2_J] * iA;
    o[26] = C[OR_S_T2_P] * iA;
    o[27] = nu * C[OR_S_T2_ETA] * iA;
    o[28] = nu * C[OR_S_T2_PHI] * iA;
}

}  // extern "C"
