// CPU oracle driver: the reference's executable restated on the CPU oracle.
// TEST INFRASTRUCTURE ONLY (the checker, and the CPU baseline of bench.py).
//
// Restates: CLI (src/init.cu:7-96), initial conditions (src/init.cu:99-378), the time
// loop with adaptive dt, output scheduling and diagnostics (src/main.cu:13-755), the
// scheduling helpers (src/io.cu:93-178) and the profiles CSV (src/io.cu:262-312).
// Snapshots are written in the raw side format "bin" (the reference declares SNAP_BIN
// at src/io.cuh:28 but never implements it); see nse2d-channel-gpu_b200/host/snapshot.h
// for the layout, which both writers follow.
#include "nse2d_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <random>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace {
constexpr double kPi = 3.14159265358979323846264338327950288;

struct Cli {
    or_config c{};
    std::string stretch = "none", init = "load", load_path, snap_fields = "all", outdir = "out", snap_fmt = "bin";
    double amp = 0.5, alpha = 1.2, phase = 0.0, rand_amp = 0.0;
    int my = 1;
    unsigned long long seed = 123456789ULL;
    int rand_nx = 48, rand_mymax = 8;
    double rand_k0 = 0.0, rand_sigma = 0.6, rand_amp_abs = 0.0;
    int statsEvery = 50, profilesWriteEvery = 0, threads = 0;
    double snap_save = 0.1, diag_save = 0.2;
    long max_steps = -1;
};

// src/common.cuh:42-114 defaults, src/init.cu:15-19 defaults, src/init.cu:20-95 parsing
Cli parse(int argc, char** argv) {
    Cli a;
    or_config& c = a.c;
    c.Nx = 1024; c.Ny = 1025; c.Lx = 12.566370612; c.h = 1.0;
    c.stretch = 0; c.beta = 0.0; c.Ub = 1.0; c.Reb = 10000.0; c.nu_override = -1;
    c.dt_init = 1e-3; c.dt_max = 1e-2; c.cfl = 0.5; c.cvisc = 0.5; c.adapt = 1; c.t_end = 200.0;
    c.F0 = 0.0; c.nforce = 1; c.lin_drag = 0.0; c.free_slip = 0;
    c.mms = 0; c.mms_A0 = 1e-3; c.mms_eps = 0.1; c.mms_Om = 1.0; c.mms_kx = 1; c.closure_diag = 0;
    for (int i = 1; i < argc; i++) {
        auto eq = [&](const char* s) { return std::strcmp(argv[i], s) == 0; };
        auto has = [&]() { return i + 1 < argc; };
        if (eq("--Nx") && has()) c.Nx = std::atoi(argv[++i]);
        else if (eq("--Ny") && has()) c.Ny = std::atoi(argv[++i]);
        else if (eq("--Lx") && has()) c.Lx = std::atof(argv[++i]);
        else if (eq("--h") && has()) c.h = std::atof(argv[++i]);
        else if (eq("--Ub") && has()) c.Ub = std::atof(argv[++i]);
        else if (eq("--Reb") && has()) c.Reb = std::atof(argv[++i]);
        else if (eq("--dt") && has()) c.dt_init = std::atof(argv[++i]);
        else if (eq("--dtmax") && has()) c.dt_max = std::atof(argv[++i]);
        else if (eq("--cfl") && has()) c.cfl = std::atof(argv[++i]);
        else if (eq("--cvisc") && has()) c.cvisc = std::atof(argv[++i]);
        else if (eq("--no-adapt")) c.adapt = 0;
        else if (eq("--tend") && has()) c.t_end = std::atof(argv[++i]);
        else if (eq("--F0") && has()) c.F0 = std::atof(argv[++i]);
        else if (eq("--nforce") && has()) c.nforce = std::atoi(argv[++i]);
        else if (eq("--drag") && has()) c.lin_drag = std::atof(argv[++i]);
        else if (eq("--nu") && has()) c.nu_override = std::atof(argv[++i]);
        else if (eq("--stretch") && has()) a.stretch = argv[++i];
        else if (eq("--beta") && has()) c.beta = std::atof(argv[++i]);
        else if (eq("--init") && has()) a.init = argv[++i];
        else if (eq("--amp") && has()) a.amp = std::atof(argv[++i]);
        else if (eq("--alpha") && has()) a.alpha = std::atof(argv[++i]);
        else if (eq("--my") && has()) a.my = std::atoi(argv[++i]);
        else if (eq("--phase") && has()) a.phase = std::atof(argv[++i]);
        else if (eq("--rand_amp") && has()) a.rand_amp = std::atof(argv[++i]);
        else if (eq("--seed") && has()) a.seed = std::stoull(argv[++i]);
        else if (eq("--load_path") && has()) a.load_path = argv[++i];
        else if (eq("--rand_nx") && has()) a.rand_nx = std::atoi(argv[++i]);
        else if (eq("--rand_mymax") && has()) a.rand_mymax = std::atoi(argv[++i]);
        else if (eq("--rand_k0") && has()) a.rand_k0 = std::atof(argv[++i]);
        else if (eq("--rand_sigma") && has()) a.rand_sigma = std::atof(argv[++i]);
        else if (eq("--rand_amp_abs") && has()) a.rand_amp_abs = std::atof(argv[++i]);
        else if (eq("--mms")) {
            c.mms = 1;
            if (i + 1 < argc && argv[i + 1][0] != '-') c.mms = (std::atoi(argv[++i]) != 0);
        }
        else if (eq("--mmsA0") && has()) c.mms_A0 = std::atof(argv[++i]);
        else if (eq("--mmsEps") && has()) c.mms_eps = std::atof(argv[++i]);
        else if (eq("--mmsOm") && has()) c.mms_Om = std::atof(argv[++i]);
        else if (eq("--mmsKx") && has()) c.mms_kx = std::atoi(argv[++i]);
        else if (eq("--statsEvery") && has()) a.statsEvery = std::atoi(argv[++i]);
        else if (eq("--closure_diag")) c.closure_diag = 1;
        else if (eq("--profilesWriteEvery") && has()) a.profilesWriteEvery = std::atoi(argv[++i]);
        else if (eq("--snap_save") && has()) a.snap_save = std::atof(argv[++i]);
        else if (eq("--snap_fmt") && has()) a.snap_fmt = argv[++i];
        else if (eq("--snap_fields") && has()) a.snap_fields = argv[++i];
        else if ((eq("--diag_save") || eq("--diagsave")) && has()) a.diag_save = std::atof(argv[++i]);
        else if (eq("--outdir") && has()) a.outdir = argv[++i];
        // oracle-only switches
        else if (eq("--free_slip")) c.free_slip = 1;
        else if (eq("--threads") && has()) a.threads = std::atoi(argv[++i]);
        else if (eq("--max_steps") && has()) a.max_steps = std::atol(argv[++i]);
    }
    if (a.init == "laminar" && a.rand_amp > 0.0 && a.amp <= 0.0) { a.init = "rand"; a.amp = a.rand_amp; }
    if (a.init == "mms") c.mms = 1;
    c.stretch = (a.stretch == "tanh") ? 1 : 0;
    return a;
}

// ---- initial conditions: src/init.cu:99-378 (load handled by the bin reader) ----
std::vector<double> initial_omega(const Cli& a, const double* y) {
    const or_config& c = a.c;
    const int Nx = c.Nx, Ny = c.Ny;
    const double Lx = c.Lx, h = c.h, Ub = c.Ub;
    std::vector<double> w((size_t)Nx * Ny, 0.0);
    auto at = [&](int j, int i) -> double& { return w[(size_t)j * Nx + i]; };
    if (a.init == "mms") {                                                       // init.cu:118-137
        const double k = (2.0 * kPi) * (double)c.mms_kx / Lx, cc = kPi / (2.0 * h), A0 = c.mms_A0;
        for (int j = 0; j < Ny; ++j) {
            const double theta = cc * (y[j] + h);
            double s = std::sin(theta); s *= s;
            const double cos2 = std::cos(2.0 * theta);
            const double g = (k * k) * s - 2.0 * (cc * cc) * cos2;
            for (int i = 0; i < Nx; ++i) at(j, i) = A0 * std::sin(k * ((double)i * (Lx / (double)Nx))) * g;
        }
        return w;
    }
    if (a.init == "diffusion") {                                                 // init.cu:151-171
        const int my0 = (a.my > 0 ? a.my : 1);
        const int n = 2 * my0;
        const double mu = (double)n * kPi / (2.0 * h);
        const double Au = (a.amp != 0.0) ? a.amp : 1.0;
        for (int j = 0; j < Ny; ++j) {
            const double wj = -Au * mu * std::cos(mu * (y[j] + h));
            for (int i = 0; i < Nx; ++i) at(j, i) = wj;
        }
        return w;
    }
    if (a.init == "diffusion2d") {                                               // init.cu:173-204
        const double alpha = (a.alpha > 0.0) ? a.alpha : (2.0 * kPi * 1.0 / Lx);
        const double beta = (double)(a.my > 0 ? a.my : 1) * kPi / (2.0 * h);
        const double lambda = alpha * alpha + beta * beta;
        const double Apsi = (a.amp != 0.0) ? a.amp : 1.0;
        for (int j = 0; j < Ny; ++j) {
            const double sj = std::sin(beta * (y[j] + h));
            for (int i = 0; i < Nx; ++i) {
                const double x = (double)i * (Lx / (double)Nx);
                at(j, i) = lambda * (Apsi * std::sin(alpha * x) * sj);
            }
        }
        return w;
    }
    unsigned long long seed = a.seed;                                            // init.cu:207-212
    auto rnd01 = [&]() { seed = 6364136223846793005ULL * seed + 1ULL; return ((seed >> 11) * 1.1102230246251565e-16); };
    for (int j = 0; j < Ny; ++j) {                                               // init.cu:285-288
        const double wj = 3.0 * Ub * y[j] / (h * h);
        for (int i = 0; i < Nx; ++i) at(j, i) = wj;
    }
    if (a.init == "mix") {                                                       // init.cu:290-296
        const double scale = std::max(1e-12, a.amp) * (Ub / h);
        for (size_t idx = 0; idx < w.size(); ++idx) w[idx] += scale * (rnd01() - 0.5);
    }
    if (a.init == "ts" || a.init == "mix") {                                     // init.cu:299-312
        const double alpha = (a.alpha > 0 ? a.alpha : (2.0 * kPi / Lx));
        const double mu = kPi * (double)a.my / (2.0 * h);
        const double Apsi = (a.amp * Ub) / std::max(1e-12, mu);
        for (int j = 0; j < Ny; ++j) {
            const double sy = std::sin(mu * (y[j] + h));
            for (int i = 0; i < Nx; ++i) {
                const double x = (double)i * (Lx / (double)Nx);
                const double psi_p = Apsi * sy * std::cos(alpha * x + a.phase);
                at(j, i) += (alpha * alpha + mu * mu) * psi_p;
            }
        }
    }
    if (a.init == "rand") {                                                      // init.cu:314-362
        const double dx = Lx / (double)Nx;
        const double alpha_min = 2.0 * kPi / Lx, alpha_nyq = kPi / dx, alpha_max = 0.35 * alpha_nyq;
        const int nxm = std::max(1, a.rand_nx), mymx = std::max(1, a.rand_mymax);
        const double k0 = (a.rand_k0 > 0 ? a.rand_k0 : (6.0 * 2.0 * kPi / Lx));
        const double sig = std::max(0.05, a.rand_sigma);
        std::mt19937_64 rng(a.seed);
        std::uniform_real_distribution<double> U01(0.0, 1.0);
        std::normal_distribution<double> N0(0.0, 1.0);
        auto sample_alpha = [&]() {
            double al = std::exp(std::log(k0) + sig * N0(rng));
            if (al < alpha_min) al = alpha_min;
            if (al > alpha_max) al = alpha_max;
            return al;
        };
        const double A0 = std::max(1e-12, (a.rand_amp_abs > 0 ? a.rand_amp_abs : a.amp)) / std::sqrt((double)nxm);
        std::vector<std::vector<double>> sY(mymx + 1, std::vector<double>(Ny, 0.0));
        for (int my = 1; my <= mymx; ++my) {
            const double mu = kPi * (double)my / (2.0 * h);
            for (int j = 0; j < Ny; ++j) sY[my][j] = std::sin(mu * (y[j] + h));
        }
        for (int m = 0; m < nxm; ++m) {
            const double alpha = sample_alpha();
            const int my = 1 + (int)std::floor(U01(rng) * mymx);
            const double phi = 2.0 * kPi * U01(rng);
            const double mu = kPi * (double)my / (2.0 * h);
            const double k = std::sqrt(alpha * alpha + mu * mu);
            const double wamp = A0 * std::exp(-0.5 * std::pow(std::log(k / k0) / sig, 2));
            for (int j = 0; j < Ny; ++j) {
                const double sj = sY[my][j];
                for (int i = 0; i < Nx; ++i) {
                    const double x = ((double)i * (Lx / (double)Nx));
                    at(j, i) += wamp * std::cos(alpha * x + phi) * sj;
                }
            }
        }
    }
    return w;
}

// ---- scheduling helpers: src/io.cu:93-178 ----
double time_tol(double t) { return 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, std::fabs(t)); }
double sched_tol(double t, double dt) { return std::max(time_tol(t), 1e-6 * std::max(1e-300, std::fabs(dt))); }

void ensure_dir(const std::string& p) {
    if (p.empty()) return;
    struct stat st;
    if (::stat(p.c_str(), &st) == 0) return;
    size_t pos = p.find_last_of('/');
    if (pos != std::string::npos && pos > 0) ensure_dir(p.substr(0, pos));
    ::mkdir(p.c_str(), 0755);
}

bool file_nonempty(const std::string& path) {
    std::ifstream f(path, std::ios::ate | std::ios::binary);
    return f.good() && f.tellg() > 0;
}

void write_snapshot_bin(const std::string& outdir, const Cli& a, or_solver* s, double t, double nu) {
    const int Nx = a.c.Nx, Ny = a.c.Ny;
    const size_t N = (size_t)Nx * Ny;
    std::string sdir = outdir + "/snaps";
    ensure_dir(sdir);
    std::ostringstream fn; fn << sdir << "/snap_t" << std::fixed << std::setprecision(6) << t << ".bin";
    std::vector<double> w(N), psi(N), u, v;
    or_get_fields(s, w.data(), psi.data());
    const bool want_psi = (a.snap_fields == "all" || a.snap_fields == "omega_psi");
    const bool want_uv = (a.snap_fields == "all");
    if (want_uv) {
        u.resize(N); v.resize(N);
        const double dx = a.c.Lx / Nx, deta = 2.0 / (Ny - 1);
        or_uv_from_psi(psi.data(), u.data(), v.data(), Nx, Ny, 1.0 / dx, 1.0 / deta, or_metric(s, 1));
    }
    FILE* f = std::fopen(fn.str().c_str(), "wb");
    if (!f) return;
    const char magic[8] = {'N', 'S', 'E', '2', 'D', 'S', 'N', 'P'};
    int32_t hdr[4] = {1, Nx, Ny, 1 + (want_psi ? 1 : 0) + (want_uv ? 2 : 0)};
    const double stretch_code = (a.stretch != "none" && a.c.beta > 0.0 && a.stretch == "tanh") ? 1.0 : 0.0;
    const int32_t has_y = (a.stretch != "none" && a.c.beta > 0.0) ? 1 : 0;
    double d[9] = {t, a.c.Lx, 2.0 * a.c.h, a.c.h, a.c.Lx / Nx, (2.0 * a.c.h) / (Ny - 1), nu, a.c.beta, stretch_code};
    std::fwrite(magic, 1, 8, f); std::fwrite(hdr, 4, 4, f); std::fwrite(d, 8, 9, f); std::fwrite(&has_y, 4, 1, f);
    auto put = [&](const char* name, const std::vector<double>& x) {
        char nm[16] = {0}; std::strncpy(nm, name, 15);
        std::fwrite(nm, 1, 16, f); std::fwrite(x.data(), 8, N, f);
    };
    put("omega", w);
    if (want_psi) put("psi", psi);
    if (want_uv) { put("u", u); put("v", v); }
    if (has_y) std::fwrite(or_metric(s, 0), 8, Ny, f);
    std::fclose(f);
}

bool read_snapshot_bin(const std::string& path, int Nx, int Ny, std::vector<double>& w, double* t) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char magic[8]; int32_t hdr[4]; double d[9]; int32_t has_y;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "NSE2DSNP", 8) == 0 &&
              std::fread(hdr, 4, 4, f) == 4 && std::fread(d, 8, 9, f) == 9 && std::fread(&has_y, 4, 1, f) == 1 &&
              hdr[1] == Nx && hdr[2] == Ny;
    if (ok) {
        char nm[16];
        ok = std::fread(nm, 1, 16, f) == 16 && std::strcmp(nm, "omega") == 0;
        w.resize((size_t)Nx * Ny);
        ok = ok && std::fread(w.data(), 8, w.size(), f) == w.size();
        if (t) *t = d[0];
    }
    std::fclose(f);
    return ok;
}

void write_profiles(const std::string& path, const Cli& a, const double* y, const double* a_node, double nu,
                    double utau, double T, const std::vector<double>* H) {       // io.cu:262-312
    const int Ny = a.c.Ny;
    const double h = a.c.h, dyu = (2.0 * h) / (Ny - 1);
    const bool mapped = (a.stretch != "none" && a.c.beta > 0.0);
    std::ofstream f(path, std::ios::out);
    f << "j,y,yplus,U,V,uu,vv,uv,Uplus,tau_total\n";
    for (int j = 0; j < Ny; ++j) {
        const double yy = mapped ? y[j] : (-h + (double)j * dyu);
        const double ybot = yy + h;
        const double Ub = (T > 0 ? H[0][j] / T : 0.0), Vb = (T > 0 ? H[1][j] / T : 0.0);
        const double U2 = (T > 0 ? H[2][j] / T : 0.0), V2 = (T > 0 ? H[3][j] / T : 0.0), UV = (T > 0 ? H[4][j] / T : 0.0);
        const double uu = std::fmax(0.0, U2 - Ub * Ub), vv = std::fmax(0.0, V2 - Vb * Vb), uv = UV - Ub * Vb;
        const double Ujp = (T > 0 ? H[0][std::min(j + 1, Ny - 1)] / T : 0.0);
        const double Ujm = (T > 0 ? H[0][std::max(j - 1, 0)] / T : 0.0);
        double dUdy;
        if (mapped) {
            const double inv_deta = (Ny > 1) ? (0.5 * (Ny - 1)) : 0.0;
            const double an = a_node[j];
            if (j == 0) dUdy = an * (Ujp - Ub) * inv_deta;
            else if (j == Ny - 1) dUdy = an * (Ub - Ujm) * inv_deta;
            else dUdy = an * (Ujp - Ujm) * 0.5 * inv_deta;
        } else {
            if (j == 0) dUdy = (Ujp - Ub) / dyu;
            else if (j == Ny - 1) dUdy = (Ub - Ujm) / dyu;
            else dUdy = (Ujp - Ujm) * 0.5 / dyu;
        }
        const double tau = nu * dUdy - uv;
        const double yplus = (utau > 0 ? utau * ybot / nu : 0.0);
        const double Uplus = (utau > 0 ? Ub / utau : 0.0);
        f.setf(std::ios::scientific); f.precision(8);
        f << j << "," << yy << "," << yplus << "," << Ub << "," << Vb << "," << uu << "," << vv << "," << uv << ","
          << Uplus << "," << tau << "\n";
    }
}

void write_row(std::ofstream& f, long step, double t, double dt, const double* v, bool closure) {
    f.setf(std::ios::scientific); f.precision(8);
    f << step << "," << t << "," << dt;
    for (int q = 0; q < 16; ++q) f << "," << v[q];
    if (closure) for (int q = 16; q < 29; ++q) f << "," << v[q];
    f << "\n";
}
}  // namespace

int main(int argc, char** argv) {
    Cli a = parse(argc, argv);
    if (a.threads > 0) or_set_threads(a.threads);
    ensure_dir(a.outdir);
    const std::string diag_path = a.outdir + "/diagnostics.csv", prof_path = a.outdir + "/profiles_timeavg.csv";
    or_solver* s = or_create(&a.c);
    if (!s) { std::fprintf(stderr, "oracle: bad configuration\n"); return 1; }
    const int Nx = a.c.Nx, Ny = a.c.Ny;
    const double nu = or_nu(s);
    const double* y = or_metric(s, 0);
    const double* a_node = or_metric(s, 1);
    const double dx = a.c.Lx / Nx, deta = 2.0 / (Ny - 1), inv_dx = 1.0 / dx, inv_deta = 1.0 / deta;

    std::vector<double> w0;
    if (a.init == "load") {
        if (!read_snapshot_bin(a.load_path, Nx, Ny, w0, nullptr)) {
            std::fprintf(stderr, "oracle: --init load needs a bin snapshot of the same grid (--load_path)\n");
            return 1;
        }
    } else {
        w0 = initial_omega(a, y);
    }
    or_set_omega(s, w0.data());

    if (!file_nonempty(diag_path)) {
        std::ofstream f(diag_path);
        f << "step,t,dt,umax,vmax,K,Omega,dOmega_rhs,eta,BOmega_wall,Pin,epsilon,POmega,tauw_bot,tauw_top,dpdx,utau_avg,Cf,Re_tau";
        if (a.c.closure_diag) f << ",dOmega_rhs_same,dOmega_rhs_same_int,Omega_int,eta_int,Jwall_s1_cum,Jwall_s2_cum,Jwall_s3_cum,Omega_int_w,dOmega_same_int_w,A_w,P_int_w,eta_h,Phi_h";
        f << "\n";
    }
    { std::ofstream f(prof_path); f << "j,y,yplus,U,V,uu,vv,uv,Uplus,tau_total\n"; }

    const bool use_snap = a.snap_save > 0, use_diag = a.diag_save > 0;
    double next_snap = use_snap ? 0.0 : 1e300, next_diag = use_diag ? 0.0 : 1e300;
    double tauw_abs_dt_sum = 0.0, T_diag = 0.0, last_diag_t = 0.0;
    double row[29];
    if (use_snap) { write_snapshot_bin(a.outdir, a, s, 0.0, nu); next_snap = a.snap_save; }
    if (use_diag) {
        or_diag_row(s, 0.0, 1, row);
        std::ofstream f(diag_path, std::ios::app);
        write_row(f, 0, 0.0, a.c.dt_init, row, a.c.closure_diag);
        next_diag = a.diag_save;
    }
    std::vector<double> H[5];
    for (auto& v : H) v.assign(Ny, 0.0);
    std::vector<double> su(Ny), sv(Ny), su2(Ny), sv2(Ny), suv(Ny);
    double T_accum = 0.0, last_stats_t = 0.0;
    double t = 0.0, dt = a.c.dt_init;
    long step = 0;
    const auto wall0 = std::chrono::steady_clock::now();
    while (t < a.c.t_end - 0.5 * dt) {                                          // main.cu:434
        if (a.max_steps >= 0 && step >= a.max_steps) break;
        if (a.c.adapt) dt = or_adapt_dt(s, nullptr);                            // main.cu:439-464
        if (a.c.adapt && (use_snap || use_diag)) {                              // main.cu:467-480
            double t_next = 1e300;
            if (use_snap) t_next = std::min(t_next, next_snap);
            if (use_diag) t_next = std::min(t_next, next_diag);
            if (t_next < 1e299) {
                const double rem = t_next - t;
                const double tol = std::max(time_tol(t_next), 1e-6 * dt);
                if (rem > tol && rem < 0.5 * dt) dt = rem;
            }
        }
        or_step(s, t, dt);
        t += dt; step++;
        if (use_snap && std::fabs(t - next_snap) <= sched_tol(t, dt)) t = next_snap;   // main.cu:544-551
        if (use_diag && std::fabs(t - next_diag) <= sched_tol(t, dt)) t = next_diag;
        if (use_snap) {                                                          // main.cu:553-563
            while (t + sched_tol(t, dt) >= next_snap && next_snap <= a.c.t_end + sched_tol(a.c.t_end, dt)) {
                write_snapshot_bin(a.outdir, a, s, next_snap, nu);
                next_snap += a.snap_save;
            }
        }
        if (use_diag && (t + time_tol(t) >= next_diag)) {                       // main.cu:566-692
            double dtw = next_diag - last_diag_t; if (dtw < 0) dtw = 0;
            last_diag_t = next_diag;
            or_diag_row(s, t, 0, row);
            const double tb = row[10], tt = row[11];
            if (dtw > 0) { tauw_abs_dt_sum += 0.5 * (std::fabs(tb) + std::fabs(tt)) * dtw; T_diag += dtw; }
            std::ofstream f(diag_path, std::ios::app);
            write_row(f, step, t, dt, row, a.c.closure_diag);
            next_diag += a.diag_save;
        }
        if (step % a.statsEvery == 0) {                                          // main.cu:695-733
            const double dtw = t - last_stats_t;
            if (dtw > 0) {
                std::vector<double> w(Nx * (size_t)Ny), psi(Nx * (size_t)Ny);
                or_get_fields(s, nullptr, psi.data());
                or_row_moments(psi.data(), Nx, Ny, inv_dx, inv_deta, a_node, su.data(), sv.data(), su2.data(), sv2.data(), suv.data());
                for (int j = 0; j < Ny; ++j) {
                    H[0][j] += su[j] / Nx * dtw; H[1][j] += sv[j] / Nx * dtw;
                    H[2][j] += su2[j] / Nx * dtw; H[3][j] += sv2[j] / Nx * dtw; H[4][j] += suv[j] / Nx * dtw;
                }
                T_accum += dtw; last_stats_t = t;
            }
        }
    }
    double utau_mean;
    if (T_diag > 0) utau_mean = std::sqrt(tauw_abs_dt_sum / T_diag);
    else {
        or_diag_row(s, t, 1, row);
        utau_mean = std::sqrt(0.5 * (std::fabs(row[10]) + std::fabs(row[11])));
    }
    write_profiles(prof_path, a, y, a_node, nu, utau_mean, T_accum, H);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    std::ofstream p(a.outdir + "/progress.log", std::ios::app);
    p << "oracle done: steps=" << step << " t=" << t << " wall_s=" << wall << " threads=" << or_get_threads() << "\n";
    or_destroy(s);
    return 0;
}
