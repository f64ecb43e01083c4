// Binary snapshot files (the "bin" format): the fields and metadata of the reference's HDF5
// snapshots (src/io.cu:183-259) in a flat little-endian layout, written and read without
// libhdf5. The reference declares a bin format (SNAP_BIN, src/io.cuh:28) but never writes one;
// this is the layout used here and by the CPU oracle:
//
//   char[8]    "NSE2DSNP"
//   int32[4]   version (1), Nx, Ny, number of fields F
//   float64[9] t, Lx, Ly = 2h, h, dx, dy = 2h/(Ny-1), nu, beta, stretch (1 tanh, 0 none)
//   int32      has_y (1 when the y coordinates follow the fields)
//   F times:   char[16] name (NUL padded: omega, psi, u, v), float64[Ny][Nx] values
//   float64[Ny] y, when has_y
#pragma once
#include <string>
#include <vector>

namespace nse2d_host {

struct Snapshot {
    int Nx = 0, Ny = 0;
    double t = 0, Lx = 0, h = 1, nu = 0, beta = 0;
    bool tanh = false;
    std::vector<std::string> names;
    std::vector<std::vector<double>> fields;
    std::vector<double> y;                       // empty when the grid is uniform
    const std::vector<double>* field(const std::string& name) const;
};

bool write_snapshot(const std::string& path, const Snapshot& s, std::string& err);
bool read_snapshot(const std::string& path, Snapshot& s, std::string& err);

}  // namespace nse2d_host
