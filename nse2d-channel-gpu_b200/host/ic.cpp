// Initial vorticity fields, restating src/init.cu:99-378 of the reference: the same formulas,
// the same random streams (a 64-bit LCG for mix, std::mt19937_64 with libstdc++'s
// normal_distribution for rand), so that the t = 0 diagnostics rows match the reference's.
#include "ic.h"

#include <algorithm>
#include <cmath>
#include <random>

namespace nse2d_host {

namespace {
constexpr double kPi = 3.14159265358979323846264338327950288;
}

bool initial_omega(const IcParams& p, const std::vector<double>& y, std::vector<double>& w, std::string& err) {
    const int Nx = p.Nx, Ny = p.Ny;
    const double Lx = p.Lx, h = p.h, Ub = p.Ub;
    w.assign((size_t)Nx * Ny, 0.0);
    auto at = [&](int j, int i) -> double& { return w[(size_t)j * Nx + i]; };
    auto xi = [&](int i) { return (double)i * (Lx / (double)Nx); };
    if (p.init == "mms") {                                                  // init.cu:118-137
        const double k = (2.0 * kPi) * (double)p.mms_kx / Lx, c = kPi / (2.0 * h);
        for (int j = 0; j < Ny; ++j) {
            const double th = c * (y[j] + h);
            double s2 = std::sin(th);
            s2 *= s2;
            const double g = (k * k) * s2 - 2.0 * (c * c) * std::cos(2.0 * th);
            for (int i = 0; i < Nx; ++i) at(j, i) = p.mms_A0 * std::sin(k * xi(i)) * g;
        }
        return true;
    }
    if (p.init == "diffusion") {                                            // init.cu:151-171
        const int n = 2 * (p.my > 0 ? p.my : 1);
        const double mu = (double)n * kPi / (2.0 * h);
        const double A = (p.amp != 0.0) ? p.amp : 1.0;
        for (int j = 0; j < Ny; ++j) {
            const double wj = -A * mu * std::cos(mu * (y[j] + h));
            for (int i = 0; i < Nx; ++i) at(j, i) = wj;
        }
        return true;
    }
    if (p.init == "diffusion2d") {                                          // init.cu:173-204
        const double al = (p.alpha > 0.0) ? p.alpha : (2.0 * kPi / Lx);
        const double be = (double)(p.my > 0 ? p.my : 1) * kPi / (2.0 * h);
        const double lam = al * al + be * be;
        const double A = (p.amp != 0.0) ? p.amp : 1.0;
        for (int j = 0; j < Ny; ++j) {
            const double sj = std::sin(be * (y[j] + h));
            for (int i = 0; i < Nx; ++i) at(j, i) = lam * (A * std::sin(al * xi(i)) * sj);
        }
        return true;
    }
    if (p.init != "laminar" && p.init != "mix" && p.init != "ts" && p.init != "rand") {
        err = "unknown --init mode '" + p.init + "'";
        return false;
    }
    for (int j = 0; j < Ny; ++j) {                                          // init.cu:285-288
        const double wj = 3.0 * Ub * y[j] / (h * h);
        for (int i = 0; i < Nx; ++i) at(j, i) = wj;
    }
    unsigned long long state = p.seed;                                      // init.cu:207-212
    auto uniform01 = [&]() {
        state = 6364136223846793005ULL * state + 1ULL;
        return (double)(state >> 11) * (1.0 / 9007199254740992.0);
    };
    if (p.init == "mix") {                                                  // init.cu:290-296
        const double scale = std::max(1e-12, p.amp) * (Ub / h);
        for (double& v : w) v += scale * (uniform01() - 0.5);
    }
    if (p.init == "ts" || p.init == "mix") {                                // init.cu:299-312
        const double al = (p.alpha > 0 ? p.alpha : (2.0 * kPi / Lx));
        const double mu = kPi * (double)p.my / (2.0 * h);
        const double Apsi = (p.amp * Ub) / std::max(1e-12, mu);
        for (int j = 0; j < Ny; ++j) {
            const double sy = std::sin(mu * (y[j] + h));
            for (int i = 0; i < Nx; ++i) at(j, i) += (al * al + mu * mu) * (Apsi * sy * std::cos(al * xi(i) + p.phase));
        }
    }
    if (p.init == "rand") {                                                 // init.cu:314-362
        const double dx = Lx / (double)Nx;
        const double a_min = 2.0 * kPi / Lx, a_max = 0.35 * (kPi / dx);
        const int nmodes = std::max(1, p.rand_nx), mymax = std::max(1, p.rand_mymax);
        const double k0 = (p.rand_k0 > 0 ? p.rand_k0 : (6.0 * 2.0 * kPi / Lx));
        const double sig = std::max(0.05, p.rand_sigma);
        std::mt19937_64 rng(p.seed);
        std::uniform_real_distribution<double> U(0.0, 1.0);
        std::normal_distribution<double> N(0.0, 1.0);
        const double A0 = std::max(1e-12, (p.rand_amp_abs > 0 ? p.rand_amp_abs : p.amp)) / std::sqrt((double)nmodes);
        std::vector<std::vector<double>> sy(mymax + 1, std::vector<double>(Ny, 0.0));
        for (int m = 1; m <= mymax; ++m)
            for (int j = 0; j < Ny; ++j) sy[m][j] = std::sin(kPi * (double)m / (2.0 * h) * (y[j] + h));
        for (int q = 0; q < nmodes; ++q) {
            double al = std::exp(std::log(k0) + sig * N(rng));
            al = std::min(std::max(al, a_min), a_max);
            const int m = 1 + (int)std::floor(U(rng) * mymax);
            const double phi = 2.0 * kPi * U(rng);
            const double mu = kPi * (double)m / (2.0 * h);
            const double k = std::sqrt(al * al + mu * mu);
            const double amp = A0 * std::exp(-0.5 * std::pow(std::log(k / k0) / sig, 2));
            for (int j = 0; j < Ny; ++j)
                for (int i = 0; i < Nx; ++i) at(j, i) += amp * std::cos(al * xi(i) + phi) * sy[m][j];
        }
    }
    return true;
}

void omega_from_psi_uniform(const IcParams& p, const std::vector<double>& psi, std::vector<double>& w) {
    const int Nx = p.Nx, Ny = p.Ny;
    const double dx = p.Lx / (double)Nx, dy = (2.0 * p.h) / (double)(Ny - 1);
    const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy);
    w.assign((size_t)Nx * Ny, 0.0);
    auto id = [&](int i, int j) { return (size_t)j * Nx + (size_t)((i + Nx) % Nx); };
    for (int j = 1; j < Ny - 1; ++j)
        for (int i = 0; i < Nx; ++i) {
            const double c = psi[id(i, j)];
            const double pxx = (psi[id(i + 1, j)] - 2 * c + psi[id(i - 1, j)]) * idx2;
            const double pyy = (psi[id(i, j + 1)] - 2 * c + psi[id(i, j - 1)]) * idy2;
            w[id(i, j)] = -(pxx + pyy);
        }
    const double pb = 0.0, pt = 2.0 * p.h * p.Ub;
    for (int i = 0; i < Nx; ++i) {
        w[id(i, 0)] = -2.0 * (psi[id(i, 1)] - pb) * idy2;
        w[id(i, Ny - 1)] = -2.0 * (psi[id(i, Ny - 2)] - pt) * idy2;
    }
}

}  // namespace nse2d_host
