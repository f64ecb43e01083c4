// Initial vorticity fields of the reference's --init modes (src/init.cu:99-378), on the host.
#pragma once
#include <string>
#include <vector>

namespace nse2d_host {

struct IcParams {
    std::string init = "laminar";      // laminar | mix | ts | rand | diffusion | diffusion2d | mms | load
    int Nx = 0, Ny = 0;
    double Lx = 0.0, h = 1.0, Ub = 1.0;
    double amp = 0.5, alpha = 1.2, phase = 0.0;
    int my = 1;
    unsigned long long seed = 123456789ULL;
    int rand_nx = 48, rand_mymax = 8;
    double rand_k0 = 0.0, rand_sigma = 0.6, rand_amp_abs = 0.0;
    double mms_A0 = 1.0;
    int mms_kx = 1;
};

// omega[Ny][Nx] for every mode but load; y are the node coordinates. Returns false (with a
// message in err) for an unknown mode.
bool initial_omega(const IcParams& p, const std::vector<double>& y, std::vector<double>& w, std::string& err);

// --load_use_psi: omega from a loaded psi by second differences on the uniform spacing
// dy = 2h/(Ny-1), walls by the first-order Thom form with psi_bot = 0, psi_top = 2 h Ub
// (src/init.cu:240-264, including its use of the uniform dy on stretched grids).
void omega_from_psi_uniform(const IcParams& p, const std::vector<double>& psi, std::vector<double>& w);

}  // namespace nse2d_host
