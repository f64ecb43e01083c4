// Snapshot files.
//
// HDF5 (the reference's format, src/io.cu:183-259, written with this project's h5lite): root
// group datasets omega, psi (--snap_fields all / omega_psi), u, v (all), each [Ny][Nx] float64;
// y [1][Ny] float64 with root attributes beta and stretch_code (1 tanh) when the grid is
// stretched; root attributes t, Nx, Ny (32-bit integers), Lx, Ly, h, dx, dy, nu (float64). Read
// back as the reference reads it (src/init.cu:215-279): omega or psi, [Ny][Nx] or its transpose.
//
// "bin": the same fields and metadata in a flat little-endian layout. The reference declares a
// bin format (SNAP_BIN, src/io.cuh:28) but never writes one; this is the layout used here and by
// the CPU oracle:
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

bool write_snapshot(const std::string& path, const Snapshot& s, std::string& err);      // bin
bool write_snapshot_h5(const std::string& path, const Snapshot& s, std::string& err);   // HDF5
// either format (told apart by the file's signature)
bool read_snapshot(const std::string& path, Snapshot& s, std::string& err);
// the dataset "y" of an HDF5 file as a vector of Ny values ([Ny][1] or [1][Ny]): --ytable
bool read_y_table(const std::string& path, int Ny, std::vector<double>& y, std::string& err);

}  // namespace nse2d_host
