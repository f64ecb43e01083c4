// nse2d: the reference's solver executable (src/main.cu:13-789, CLI src/init.cu:7-96) on the
// B200 time step, through the C ABI of libnse2d_b200.so only.
//
// Same flags, same outputs in --outdir: diagnostics.csv (with the --closure_diag columns),
// profiles_timeavg.csv (time-weighted statistics every --statsEvery steps, rolling rewrites
// every --profilesWriteEvery steps), spectra_kx.csv (--spectraEvery), timing.csv (--profile,
// every --timeEvery steps), snapshots every --snap_save and progress.log. The reference's
// free-slip executable (nse2d_freeslip, built with -DFREE_SLIP_WALLS) is this program called
// under that name, or with --free_slip.
//
// The time loop runs on the device: nse2d_run steps inside one graph launch until an output
// time, a statistics step or t_end needs the host (with --profile, one profiled step at a
// time). dt trimming, the snap to output times and the step counter are the device's.
//
// Snapshots are the reference's HDF5 files (src/io.cu:183-259, written by host/h5lite without
// libhdf5): snaps/snap_t%.6f.h5. --snap_fmt bin writes the flat "bin" layout of host/snapshot.h
// instead (the format the reference declares but never writes), --snap_fmt both writes the two.
// --init load and --resume read either (src/init.cu:215-279, src/main.cu:129-147), and
// --stretch table reads y from the HDF5 file of --ytable (src/grid.cu:46-78).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <numeric>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/nse2d.h"
#include "ic.h"
#include "snapshot.h"

using nse2d_host::IcParams;
using nse2d_host::Snapshot;

namespace {

struct Args {
    nse2d_config c{};
    IcParams ic;
    std::string stretch = "none", outdir = "out", snap_fmt = "h5", snap_fields = "all", load_path, ytable;
    bool load_use_psi = false, resume = false, profile = false;
    int statsEvery = 50, timeEvery = 50, spectraEvery = 0, profilesWriteEvery = 0;
    double snap_save = 0.1, diag_save = 0.2, rand_amp = 0.0;
};

// src/init.cu:20-95: unknown flags are ignored, as there
Args parse(int argc, char** argv) {
    Args a;
    nse2d_config_default(&a.c);
    a.ic.init = "load";
    for (int i = 1; i < argc; ++i) {
        auto eq = [&](const char* s) { return std::strcmp(argv[i], s) == 0; };
        auto has = [&]() { return i + 1 < argc; };
        nse2d_config& c = a.c;
        IcParams& p = a.ic;
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
        else if (eq("--ytable") && has()) a.ytable = argv[++i];
        else if (eq("--integrator") && has()) ++i;                  // parsed, unused (always SSPRK3)
        else if (eq("--init") && has()) p.init = argv[++i];
        else if (eq("--amp") && has()) p.amp = std::atof(argv[++i]);
        else if (eq("--alpha") && has()) p.alpha = std::atof(argv[++i]);
        else if (eq("--my") && has()) p.my = std::atoi(argv[++i]);
        else if (eq("--phase") && has()) p.phase = std::atof(argv[++i]);
        else if (eq("--rand_amp") && has()) a.rand_amp = std::atof(argv[++i]);
        else if (eq("--seed") && has()) p.seed = std::stoull(argv[++i]);
        else if (eq("--load_path") && has()) a.load_path = argv[++i];
        else if (eq("--load_use_psi")) a.load_use_psi = true;
        else if (eq("--rand_nx") && has()) p.rand_nx = std::atoi(argv[++i]);
        else if (eq("--rand_mymax") && has()) p.rand_mymax = std::atoi(argv[++i]);
        else if (eq("--rand_k0") && has()) p.rand_k0 = std::atof(argv[++i]);
        else if (eq("--rand_sigma") && has()) p.rand_sigma = std::atof(argv[++i]);
        else if (eq("--rand_amp_abs") && has()) p.rand_amp_abs = std::atof(argv[++i]);
        else if (eq("--mms")) {
            c.mms = 1;
            if (i + 1 < argc && argv[i + 1][0] != '-') c.mms = (std::atoi(argv[++i]) != 0);
        }
        else if (eq("--mmsA0") && has()) c.mms_A0 = std::atof(argv[++i]);
        else if (eq("--mmsEps") && has()) c.mms_eps = std::atof(argv[++i]);
        else if (eq("--mmsOm") && has()) c.mms_Om = std::atof(argv[++i]);
        else if (eq("--mmsKx") && has()) c.mms_kx = std::atoi(argv[++i]);
        else if (eq("--statsEvery") && has()) a.statsEvery = std::atoi(argv[++i]);
        else if (eq("--timeEvery") && has()) a.timeEvery = std::atoi(argv[++i]);
        else if (eq("--profile")) a.profile = true;
        else if (eq("--closure_diag")) c.closure_diag = 1;
        else if (eq("--resume")) a.resume = true;
        else if (eq("--profilesWriteEvery") && has()) a.profilesWriteEvery = std::atoi(argv[++i]);
        else if (eq("--snap_save") && has()) a.snap_save = std::atof(argv[++i]);
        else if (eq("--snap_fmt") && has()) a.snap_fmt = argv[++i];
        else if (eq("--snap_fields") && has()) a.snap_fields = argv[++i];
        else if ((eq("--diag_save") || eq("--diagsave")) && has()) a.diag_save = std::atof(argv[++i]);
        else if (eq("--spectraEvery") && has()) a.spectraEvery = std::atoi(argv[++i]);
        else if (eq("--outdir") && has()) a.outdir = argv[++i];
        else if (eq("--free_slip")) c.free_slip = 1;
        else if (eq("--fp32")) c.precision = 32;                      // FP32-bulk variant (this build)
    }
    if (a.ic.init == "laminar" && a.rand_amp > 0.0 && a.ic.amp <= 0.0) {   // init.cu:91-93
        a.ic.init = "rand";
        a.ic.amp = a.rand_amp;
    }
    if (a.ic.init == "mms") a.c.mms = 1;                                  // init.cu:95
    a.c.stretch = (a.stretch == "tanh") ? 1 : (a.stretch == "table") ? 2 : 0;
    a.ic.Nx = a.c.Nx; a.ic.Ny = a.c.Ny; a.ic.Lx = a.c.Lx; a.ic.h = a.c.h; a.ic.Ub = a.c.Ub;
    a.ic.mms_A0 = a.c.mms_A0; a.ic.mms_kx = a.c.mms_kx;
    return a;
}

// src/io.cu:158-178
double time_tol(double t) { return 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, std::fabs(t)); }
double sched_tol(double t, double dt) { return std::max(time_tol(t), 1e-6 * std::max(1e-300, std::fabs(dt))); }
double next_after(double t0, double dt) {
    if (dt <= 0.0) return 1e300;
    const double k = std::floor((t0 + time_tol(t0)) / dt);
    const double t1 = (k + 1.0) * dt;
    return (t1 <= t0 + time_tol(t0)) ? t1 + dt : t1;
}

void ensure_dir(const std::string& p) {
    if (p.empty()) return;
    struct stat st;
    if (::stat(p.c_str(), &st) == 0) return;
    const size_t pos = p.find_last_of('/');
    if (pos != std::string::npos && pos > 0) ensure_dir(p.substr(0, pos));
    ::mkdir(p.c_str(), 0755);
}

bool file_nonempty(const std::string& path) {
    std::ifstream f(path, std::ios::ate | std::ios::binary);
    return f.good() && f.tellg() > 0;
}

class Log {
  public:
    explicit Log(const std::string& path) : path_(path) {}
    void operator()(const char* fmt, ...) {
        char buf[2048];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        std::fputs(buf, stdout);
        std::ofstream f(path_, std::ios::app);
        f << buf;
    }

  private:
    std::string path_;
};

struct Run {
    Args a;
    nse2d_ctx* ctx = nullptr;
    int Nx = 0, Ny = 0;
    double nu = 0.0;
    std::vector<double> y, a_node;
    bool mapped = false;
};

int fail(const char* what) {
    std::fprintf(stderr, "nse2d: %s: %s\n", what, nse2d_last_error());
    return 1;
}

bool write_snap(Run& r, double t, std::string& err) {
    const Args& a = r.a;
    const size_t N = (size_t)r.Nx * r.Ny;
    Snapshot s;
    s.Nx = r.Nx; s.Ny = r.Ny; s.t = t; s.Lx = a.c.Lx; s.h = a.c.h; s.nu = r.nu; s.beta = a.c.beta;
    s.tanh = r.mapped && a.stretch == "tanh";
    std::vector<double> w(N), psi(N);
    if (nse2d_get_fields(r.ctx, w.data(), psi.data(), 0, nullptr)) { err = nse2d_last_error(); return false; }
    s.names.push_back("omega");
    s.fields.push_back(std::move(w));
    if (a.snap_fields == "all" || a.snap_fields == "omega_psi") {
        s.names.push_back("psi");
        s.fields.push_back(std::move(psi));
    }
    if (a.snap_fields == "all") {
        double *du = nullptr, *dv = nullptr;
        std::vector<double> u(N), v(N);
        if (nse2d_field_ptr(r.ctx, 2, &du) || nse2d_field_ptr(r.ctx, 3, &dv) || nse2d_uv(r.ctx, du, dv, nullptr) ||
            nse2d_get_field(r.ctx, 2, u.data(), nullptr) || nse2d_get_field(r.ctx, 3, v.data(), nullptr)) {
            err = nse2d_last_error();
            return false;
        }
        s.names.push_back("u");
        s.fields.push_back(std::move(u));
        s.names.push_back("v");
        s.fields.push_back(std::move(v));
    }
    if (r.mapped) s.y = r.y;
    ensure_dir(a.outdir + "/snaps");
    std::ostringstream fn;
    fn << a.outdir << "/snaps/snap_t" << std::fixed << std::setprecision(6) << t;
    // the reference maps every --snap_fmt value to HDF5 (src/main.cu:126-127); bin and both are this
    // build's additions
    const bool bin = a.snap_fmt == "bin" || a.snap_fmt == "both", h5 = a.snap_fmt != "bin";
    if (h5 && !nse2d_host::write_snapshot_h5(fn.str() + ".h5", s, err)) return false;
    if (bin && !nse2d_host::write_snapshot(fn.str() + ".bin", s, err)) return false;
    return true;
}

void write_row(const std::string& path, long long step, double t, double dt, const double* v, bool closure) {
    std::ofstream f(path, std::ios::app);
    f.setf(std::ios::scientific);
    f.precision(8);
    f << step << "," << t << "," << dt;
    for (int q = 0; q < 16; ++q) f << "," << v[q];
    if (closure)
        for (int q = 16; q < 29; ++q) f << "," << v[q];
    f << "\n";
}

// src/io.cu:262-312
void write_profiles(const Run& r, const std::string& path, double utau, double T, const std::vector<double>* H) {
    const int Ny = r.Ny;
    const double h = r.a.c.h, dyu = (2.0 * h) / (Ny - 1);
    std::ofstream f(path, std::ios::out);
    f << "j,y,yplus,U,V,uu,vv,uv,Uplus,tau_total\n";
    f.setf(std::ios::scientific);
    f.precision(8);
    for (int j = 0; j < Ny; ++j) {
        const double yy = r.mapped ? r.y[j] : (-h + (double)j * dyu);
        const double ybot = yy + h;
        const double Ub = (T > 0 ? H[0][j] / T : 0.0), Vb = (T > 0 ? H[1][j] / T : 0.0);
        const double U2 = (T > 0 ? H[2][j] / T : 0.0), V2 = (T > 0 ? H[3][j] / T : 0.0);
        const double UV = (T > 0 ? H[4][j] / T : 0.0);
        const double uu = std::fmax(0.0, U2 - Ub * Ub), vv = std::fmax(0.0, V2 - Vb * Vb), uv = UV - Ub * Vb;
        const double Ujp = (T > 0 ? H[0][std::min(j + 1, Ny - 1)] / T : 0.0);
        const double Ujm = (T > 0 ? H[0][std::max(j - 1, 0)] / T : 0.0);
        double dUdy;
        if (r.mapped) {
            const double inv_deta = 0.5 * (Ny - 1), an = r.a_node[j];
            if (j == 0) dUdy = an * (Ujp - Ub) * inv_deta;
            else if (j == Ny - 1) dUdy = an * (Ub - Ujm) * inv_deta;
            else dUdy = an * (Ujp - Ujm) * 0.5 * inv_deta;
        } else {
            if (j == 0) dUdy = (Ujp - Ub) / dyu;
            else if (j == Ny - 1) dUdy = (Ub - Ujm) / dyu;
            else dUdy = (Ujp - Ujm) * 0.5 / dyu;
        }
        const double tau = r.nu * dUdy - uv;
        const double yplus = (utau > 0 ? utau * ybot / r.nu : 0.0);
        const double Uplus = (utau > 0 ? Ub / utau : 0.0);
        f << j << "," << yy << "," << yplus << "," << Ub << "," << Vb << "," << uu << "," << vv << "," << uv << ","
          << Uplus << "," << tau << "\n";
    }
}

// u_tau of the current state from the wall shear stresses (the tauw columns of a t = 0 style
// row: src/main.cu:702-711)
double utau_now(Run& r) {
    double row[29];
    if (nse2d_diagnostics(r.ctx, 1, row, nullptr)) return 0.0;
    return std::sqrt(0.5 * (std::fabs(row[10]) + std::fabs(row[11])));
}

}  // namespace

int main(int argc, char** argv) {
    Run r;
    r.a = parse(argc, argv);
    Args& a = r.a;
    const std::string prog = argv[0];
    if (prog.size() >= 8 && prog.find("freeslip") != std::string::npos) a.c.free_slip = 1;
    ensure_dir(a.outdir);
    Log LOGP(a.outdir + "/progress.log");
    std::vector<double> ytab;
    if (a.stretch == "table") {                                                 // grid.cu:46-78
        std::string terr;
        if (a.ytable.empty()) { std::fprintf(stderr, "nse2d: --ytable required for --stretch table\n"); return 1; }
        if (!nse2d_host::read_y_table(a.ytable, a.c.Ny, ytab, terr)) {
            std::fprintf(stderr, "nse2d: %s: %s\n", a.ytable.c_str(), terr.c_str());
            return 1;
        }
        a.c.y_table = ytab.data();
    } else if (a.stretch != "none" && a.stretch != "uniform" && a.stretch != "tanh") {
        std::fprintf(stderr, "nse2d: Unknown --stretch '%s'\n", a.stretch.c_str());
        return 1;
    }
    if (nse2d_create(&a.c, &r.ctx)) return fail("configuration");
    r.Nx = a.c.Nx; r.Ny = a.c.Ny;
    r.mapped = (a.stretch != "none" && a.c.beta > 0.0);
    r.y.resize(r.Ny); r.a_node.resize(r.Ny);
    nse2d_metrics(r.ctx, 0, r.y.data());
    nse2d_metrics(r.ctx, 1, r.a_node.data());
    nse2d_scalar(r.ctx, 0, &r.nu);
    const size_t N = (size_t)r.Nx * r.Ny;
    const std::string diag_path = a.outdir + "/diagnostics.csv", prof_path = a.outdir + "/profiles_timeavg.csv";
    const std::string time_path = a.outdir + "/timing.csv";

    // initial condition (src/init.cu:99-378, src/main.cu:129-147, 197-215)
    double t_start = 0.0;
    std::vector<double> w0;
    std::string err;
    if (a.ic.init == "load" || a.resume) {
        if (a.load_path.empty()) {
            std::fprintf(stderr, "nse2d: %s needs --load_path /path/to/snap_tXXXXXX.h5\n",
                         a.resume ? "--resume" : "--init load");
            return 1;
        }
        Snapshot s;
        if (!nse2d_host::read_snapshot(a.load_path, s, err)) { std::fprintf(stderr, "nse2d: %s\n", err.c_str()); return 1; }
        if (s.Nx != r.Nx || s.Ny != r.Ny) { std::fprintf(stderr, "nse2d: snapshot grid does not match (Nx,Ny)\n"); return 1; }
        if (std::fabs(s.Lx - a.c.Lx) > 1e-12 || std::fabs(s.h - a.c.h) > 1e-12) {
            std::fprintf(stderr, "nse2d: snapshot geometry (Lx,h) does not match the current run\n");
            return 1;
        }
        const std::vector<double>* sw = s.field("omega");
        const std::vector<double>* sp = s.field("psi");
        if (!sw && !sp) { std::fprintf(stderr, "nse2d: snapshot has neither omega nor psi\n"); return 1; }
        if (sw && !a.load_use_psi) w0 = *sw;
        else nse2d_host::omega_from_psi_uniform(a.ic, *sp, w0);
        if (a.resume) t_start = s.t;
        LOGP("Loaded IC from %s%s, nu=%g\n", a.load_path.c_str(), (sw && !a.load_use_psi) ? " (omega)" : " (psi->omega)", s.nu);
    } else if (!nse2d_host::initial_omega(a.ic, r.y, w0, err)) {
        std::fprintf(stderr, "nse2d: %s\n", err.c_str());
        return 1;
    }
    if (nse2d_set_omega(r.ctx, w0.data(), 0, nullptr)) return fail("initial state");
    if (t_start != 0.0) {
        std::vector<double> w(N), psi(N);
        if (nse2d_get_fields(r.ctx, w.data(), psi.data(), 0, nullptr) ||
            nse2d_set_state(r.ctx, w.data(), psi.data(), 0, t_start, nullptr))
            return fail("resume state");
    }

    if (!file_nonempty(diag_path)) {                                          // main.cu:160-165
        std::ofstream f(diag_path);
        f << "step,t,dt,umax,vmax,K,Omega,dOmega_rhs,eta,BOmega_wall,Pin,epsilon,POmega,tauw_bot,tauw_top,dpdx,utau_avg,Cf,Re_tau";
        if (a.c.closure_diag)
            f << ",dOmega_rhs_same,dOmega_rhs_same_int,Omega_int,eta_int,Jwall_s1_cum,Jwall_s2_cum,Jwall_s3_cum,"
                 "Omega_int_w,dOmega_same_int_w,A_w,P_int_w,eta_h,Phi_h";
        f << "\n";
    }
    if (a.profile && !file_nonempty(time_path)) { std::ofstream g(time_path); g << "step,t,dt,t_step_ms,t_fft_ms,t_tridiag_ms\n"; }
    { std::ofstream f(prof_path); f << "j,y,yplus,U,V,uu,vv,uv,Uplus,tau_total\n"; }

    if (a.resume) LOGP("[mode] Resume simulation from %s, t0=%.6f\n", a.load_path.c_str(), t_start);
    else LOGP("[mode] New simulation (fresh IC), t0=0.000000\n");
    LOGP("[params] Nx=%d Ny=%d Lx=%.6f h=%.6f Ub=%.6f Reb=%.1f nu=%.6e dt_init=%.6g cfl=%.3g adapt=%s t_end=%.6g\n",
         r.Nx, r.Ny, a.c.Lx, a.c.h, a.c.Ub, a.c.Reb, r.nu, a.c.dt_init, a.c.cfl, a.c.adapt ? "yes" : "no", a.c.t_end);
    LOGP("[integrator] SSPRK3 (fully explicit)\n");

    const bool use_snap = a.snap_save > 0, use_diag = a.diag_save > 0;
    double next_snap = use_snap ? (a.resume ? next_after(t_start, a.snap_save) : 0.0) : 1e300;
    double next_diag = use_diag ? (a.resume ? next_after(t_start, a.diag_save) : 0.0) : 1e300;
    double row[29];
    if (!a.resume && use_snap) {                                                // main.cu:318-321
        if (!write_snap(r, 0.0, err)) { std::fprintf(stderr, "nse2d: %s\n", err.c_str()); return 1; }
        next_snap = a.snap_save;
    }
    if (!a.resume && use_diag) {                                                // main.cu:322-421
        if (nse2d_diagnostics(r.ctx, 1, row, nullptr)) return fail("diagnostics");
        write_row(diag_path, 0, 0.0, a.c.dt_init, row, a.c.closure_diag);
        next_diag = a.diag_save;
    }

    std::vector<double> H[5];
    for (auto& v : H) v.assign(r.Ny, 0.0);
    std::vector<double> mom(5 * (size_t)r.Ny);
    double tauw_abs_dt_sum = 0.0, T_diag = 0.0, last_diag_t = t_start, T_accum = 0.0, last_stats_t = t_start;
    // the time-weighted statistics accumulate on the device inside the run's graph (precision 64,
    // not with --profile); the run then halts only where the host must write rolling profiles or
    // take a spectra sample
    const bool dev_stats = a.statsEvery > 0 && a.c.precision == 64 && !a.profile;
    if (dev_stats && nse2d_stats_device(r.ctx, a.statsEvery, nullptr)) return fail("statistics");
    long long every = 0;                                                       // halt cadence (0: none)
    if (a.statsEvery > 0) every = dev_stats ? 0 : a.statsEvery;
    if (dev_stats && a.profilesWriteEvery > 0) every = std::lcm((long long)a.statsEvery, (long long)a.profilesWriteEvery);
    if (a.spectraEvery > 0) every = every ? std::gcd(every, (long long)a.spectraEvery) : a.spectraEvery;
    auto device_stats = [&]() -> bool {                                         // H and T_accum from the device
        std::vector<double> acc(5 * (size_t)r.Ny);
        if (nse2d_stats_read(r.ctx, acc.data(), &T_accum, nullptr)) return false;
        for (int q = 0; q < 5; ++q)
            for (int j = 0; j < r.Ny; ++j) H[q][j] = acc[(size_t)q * r.Ny + j];
        return true;
    };
    double t = t_start, dt = a.c.dt_init;
    long long step = 0;
    const auto wall0 = std::chrono::steady_clock::now();
    LOGP("[run] t0=%.6f -> t_end=%.6f\n", t_start, a.c.t_end);
    while (t < a.c.t_end - 0.5 * dt) {                                          // main.cu:434
        if (!(dt > 0.0) && !a.c.adapt) { std::fprintf(stderr, "nse2d: dt must be positive\n"); return 1; }
        double step_ms = 0, fft_ms = 0, tri_ms = 0;
        if (a.profile) {
            if (nse2d_set_schedule(r.ctx, use_snap ? next_snap : 1e300, use_diag ? next_diag : 1e300, nullptr) ||
                nse2d_step_profiled(r.ctx, &step_ms, &fft_ms, &tri_ms, nullptr))
                return fail("step");
        } else {
            int reason = 0;
            if (nse2d_run(r.ctx, use_snap ? next_snap : 1e300, use_diag ? next_diag : 1e300, (int)every, a.c.t_end,
                          20000, &reason, nullptr))
                return fail("run");
            if (reason & NSE2D_HALT_NONFINITE) {
                int flag = 0;
                if (nse2d_nonfinite(r.ctx, &flag, nullptr)) return fail("non-finite flag");
                if (flag & 2) {
                    std::fprintf(stderr, "nse2d: a device wait timed out; stopping\n");
                    return 1;
                }
                // NaN or Inf in psi: reported once; the run goes on, as the reference's loop does
                double tn = 0.0;
                long long sn = 0;
                if (nse2d_get_time(r.ctx, &tn, nullptr, &sn, nullptr, nullptr)) return fail("time");
                LOGP("[warn] non-finite values in psi after step %lld (t=%.6f)\n", sn, tn);
            }
        }
        if (nse2d_get_time(r.ctx, &t, &dt, &step, nullptr, nullptr)) return fail("time");
        if (use_snap) {                                                         // main.cu:553-563
            while (t + sched_tol(t, dt) >= next_snap && next_snap <= a.c.t_end + sched_tol(a.c.t_end, dt)) {
                if (!write_snap(r, next_snap, err)) { std::fprintf(stderr, "nse2d: %s\n", err.c_str()); return 1; }
                next_snap += a.snap_save;
            }
        }
        if (use_diag && t + time_tol(t) >= next_diag) {                         // main.cu:566-692
            double dtw = next_diag - last_diag_t;
            if (dtw < 0) dtw = 0;
            last_diag_t = next_diag;
            if (nse2d_diagnostics(r.ctx, 0, row, nullptr)) return fail("diagnostics");
            if (dtw > 0) {
                tauw_abs_dt_sum += 0.5 * (std::fabs(row[10]) + std::fabs(row[11])) * dtw;
                T_diag += dtw;
            }
            write_row(diag_path, step, t, dt, row, a.c.closure_diag);
            next_diag += a.diag_save;
        }
        if (dev_stats && a.profilesWriteEvery > 0 && step % a.statsEvery == 0 && step % a.profilesWriteEvery == 0) {
            if (!device_stats()) return fail("statistics");                    // main.cu:722-731
            const double utau = (T_diag > 0) ? std::sqrt(tauw_abs_dt_sum / T_diag) : utau_now(r);
            write_profiles(r, prof_path, utau, T_accum, H);
        }
        if (!dev_stats && a.statsEvery > 0 && step % a.statsEvery == 0) {      // main.cu:695-733
            const double dtw = t - last_stats_t;
            if (dtw > 0) {
                if (nse2d_row_moments(r.ctx, mom.data(), nullptr)) return fail("statistics");
                for (int q = 0; q < 5; ++q)
                    for (int j = 0; j < r.Ny; ++j) H[q][j] += mom[(size_t)q * r.Ny + j] / (double)r.Nx * dtw;
                T_accum += dtw;
                last_stats_t = t;
                if (a.profilesWriteEvery > 0 && step % a.profilesWriteEvery == 0) {
                    const double utau = (T_diag > 0) ? std::sqrt(tauw_abs_dt_sum / T_diag) : utau_now(r);
                    write_profiles(r, prof_path, utau, T_accum, H);
                }
            }
        }
        if (a.spectraEvery > 0 && step % a.spectraEvery == 0)                   // main.cu:736-744
            if (nse2d_spectra_accumulate(r.ctx, nullptr)) return fail("spectra");
        if (a.profile && a.timeEvery > 0 && step % a.timeEvery == 0) {           // main.cu:746-753
            std::ofstream g(time_path, std::ios::app);
            g.setf(std::ios::scientific);
            g.precision(6);
            g << step << "," << t << "," << dt << "," << step_ms << "," << fft_ms << "," << tri_ms << "\n";
        }
    }
    if (dev_stats && !device_stats()) return fail("statistics");
    const double utau_mean = (T_diag > 0) ? std::sqrt(tauw_abs_dt_sum / T_diag) : utau_now(r);   // main.cu:756-770
    write_profiles(r, prof_path, utau_mean, T_accum, H);
    if (a.spectraEvery > 0) {                                                   // main.cu:777-780
        const int Hn = r.Nx / 2 + 1;
        std::vector<double> kx(Hn), eu(Hn), ev(Hn);
        int samples = 0;
        if (nse2d_spectra(r.ctx, kx.data(), eu.data(), ev.data(), &samples, nullptr)) return fail("spectra");
        std::ofstream f(a.outdir + "/spectra_kx.csv");
        f.setf(std::ios::scientific);
        f.precision(10);
        f << "kx,E_u,E_v,E_tot\n";
        for (int k = 0; k < Hn; ++k) f << kx[k] << "," << eu[k] << "," << ev[k] << "," << eu[k] + ev[k] << "\n";
    }
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    LOGP("[done] steps=%lld t=%.6f wall_s=%.3f steps_per_s=%.1f\n", step, t, wall, wall > 0 ? step / wall : 0.0);
    nse2d_destroy(r.ctx);
    return 0;
}
