#include "snapshot.h"

#include <cstdint>
#include <cstdio>
#include <cstring>

#include "h5lite.h"

namespace nse2d_host {

const std::vector<double>* Snapshot::field(const std::string& name) const {
    for (size_t q = 0; q < names.size(); ++q)
        if (names[q] == name) return &fields[q];
    return nullptr;
}

bool write_snapshot(const std::string& path, const Snapshot& s, std::string& err) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { err = "cannot write " + path; return false; }
    const size_t N = (size_t)s.Nx * s.Ny;
    const char magic[8] = {'N', 'S', 'E', '2', 'D', 'S', 'N', 'P'};
    const int32_t hdr[4] = {1, s.Nx, s.Ny, (int32_t)s.fields.size()};
    const double d[9] = {s.t, s.Lx, 2.0 * s.h, s.h, s.Lx / s.Nx, (2.0 * s.h) / (s.Ny - 1), s.nu, s.beta,
                         s.tanh ? 1.0 : 0.0};
    const int32_t has_y = s.y.empty() ? 0 : 1;
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(hdr, 4, 4, f) == 4 && std::fwrite(d, 8, 9, f) == 9 &&
              std::fwrite(&has_y, 4, 1, f) == 1;
    for (size_t q = 0; ok && q < s.fields.size(); ++q) {
        char nm[16] = {0};
        std::strncpy(nm, s.names[q].c_str(), 15);
        ok = std::fwrite(nm, 1, 16, f) == 16 && s.fields[q].size() == N && std::fwrite(s.fields[q].data(), 8, N, f) == N;
    }
    if (ok && has_y) ok = std::fwrite(s.y.data(), 8, s.y.size(), f) == s.y.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = "short write to " + path;
    return ok;
}

// The reference's HDF5 layout (src/io.cu:226-256): the fields, y with beta and stretch_code on a
// stretched grid, then the scalar attributes in the reference's order.
bool write_snapshot_h5(const std::string& path, const Snapshot& s, std::string& err) {
    const size_t N = (size_t)s.Nx * s.Ny;
    std::vector<h5lite::WriteDataset> ds;
    for (size_t q = 0; q < s.fields.size(); ++q) {
        if (s.fields[q].size() != N) { err = "snapshot field " + s.names[q] + " has the wrong size"; return false; }
        ds.push_back({s.names[q], {(uint64_t)s.Ny, (uint64_t)s.Nx}, s.fields[q].data()});
    }
    std::vector<h5lite::WriteAttr> at;
    auto dbl = [&](const char* n, double v) { h5lite::WriteAttr a; a.name = n; a.d = v; at.push_back(a); };
    auto i32 = [&](const char* n, int v) { h5lite::WriteAttr a; a.name = n; a.is_int = true; a.i = v; at.push_back(a); };
    if (s.tanh && s.beta > 0.0 && !s.y.empty()) {
        ds.push_back({"y", {1, (uint64_t)s.Ny}, s.y.data()});
        dbl("beta", s.beta);
        dbl("stretch_code", 1.0);
    }
    dbl("t", s.t);
    i32("Nx", s.Nx);
    i32("Ny", s.Ny);
    dbl("Lx", s.Lx);
    dbl("Ly", 2.0 * s.h);
    dbl("h", s.h);
    dbl("dx", s.Lx / (double)s.Nx);
    dbl("dy", (2.0 * s.h) / (double)(s.Ny - 1));
    dbl("nu", s.nu);
    return h5lite::write_file(path, ds, at, err);
}

static bool is_hdf5(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    unsigned char m[8] = {0};
    const bool ok = std::fread(m, 1, 8, f) == 8 && m[0] == 0x89 && std::memcmp(m + 1, "HDF\r\n\x1a\n", 7) == 0;
    std::fclose(f);
    return ok;
}

// src/init.cu:215-279: attributes Nx, Ny, Lx, h, nu, t; omega and psi as [Ny][Nx] or [Nx][Ny]
static bool read_snapshot_h5(const std::string& path, Snapshot& s, std::string& err) {
    h5lite::File f;
    if (!f.open(path, err)) return false;
    double v = 0;
    s.Nx = f.attr("Nx", v) ? (int)v : -1;
    s.Ny = f.attr("Ny", v) ? (int)v : -1;
    s.Lx = f.attr("Lx", v) ? v : -1.0;
    s.h = f.attr("h", v) ? v : -1.0;
    s.nu = f.attr("nu", v) ? v : 0.0;
    s.t = f.attr("t", v) ? v : 0.0;
    s.beta = f.attr("beta", v) ? v : 0.0;
    s.tanh = f.attr("stretch_code", v) && v == 1.0;
    if (s.Nx <= 0 || s.Ny <= 1) { err = path + ": no Nx / Ny attributes"; return false; }
    s.names.clear();
    s.fields.clear();
    for (const char* name : {"omega", "psi", "u", "v"}) {
        if (!f.has(name)) continue;
        std::vector<uint64_t> dims;
        std::vector<double> a;
        if (!f.read(name, dims, a, err)) return false;
        const uint64_t Nx = (uint64_t)s.Nx, Ny = (uint64_t)s.Ny;
        if (dims.size() == 2 && dims[0] == Ny && dims[1] == Nx) {
            s.fields.push_back(std::move(a));
        } else if (dims.size() == 2 && dims[0] == Nx && dims[1] == Ny) {      // stored [Nx][Ny]
            std::vector<double> b(a.size());
            for (uint64_t j = 0; j < Ny; ++j)
                for (uint64_t i = 0; i < Nx; ++i) b[j * Nx + i] = a[i * Ny + j];
            s.fields.push_back(std::move(b));
        } else {
            err = path + ": dataset " + name + " does not have the grid's shape";
            return false;
        }
        s.names.push_back(name);
    }
    s.y.clear();
    if (f.has("y")) {
        std::vector<uint64_t> dims;
        if (!f.read("y", dims, s.y, err)) return false;
        if ((int)s.y.size() != s.Ny) s.y.clear();
    }
    return true;
}

bool read_y_table(const std::string& path, int Ny, std::vector<double>& y, std::string& err) {
    h5lite::File f;
    if (!f.open(path, err)) return false;
    if (!f.has("y")) { err = "--ytable missing dataset /y"; return false; }
    std::vector<uint64_t> dims;
    if (!f.read("y", dims, y, err)) return false;
    const bool col = dims.size() == 2 && dims[0] == (uint64_t)Ny && dims[1] == 1;
    const bool row = dims.size() == 2 && dims[0] == 1 && dims[1] == (uint64_t)Ny;
    if (!col && !row) { err = "--ytable: could not read /y array"; return false; }
    return true;
}

bool read_snapshot(const std::string& path, Snapshot& s, std::string& err) {
    if (is_hdf5(path)) return read_snapshot_h5(path, s, err);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open snapshot " + path; return false; }
    char magic[8];
    int32_t hdr[4];
    double d[9];
    int32_t has_y = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "NSE2DSNP", 8) == 0 && std::fread(hdr, 4, 4, f) == 4 &&
              std::fread(d, 8, 9, f) == 9 && std::fread(&has_y, 4, 1, f) == 1 && hdr[0] == 1 && hdr[1] > 0 && hdr[2] > 1 &&
              hdr[3] >= 0 && hdr[3] <= 16;
    if (!ok) {
        std::fclose(f);
        err = path + " is not an NSE2DSNP snapshot";
        return false;
    }
    s.Nx = hdr[1]; s.Ny = hdr[2];
    s.t = d[0]; s.Lx = d[1]; s.h = d[3]; s.nu = d[6]; s.beta = d[7]; s.tanh = d[8] != 0.0;
    const size_t N = (size_t)s.Nx * s.Ny;
    s.names.clear();
    s.fields.clear();
    for (int q = 0; ok && q < hdr[3]; ++q) {
        char nm[17] = {0};
        std::vector<double> v(N);
        ok = std::fread(nm, 1, 16, f) == 16 && std::fread(v.data(), 8, N, f) == N;
        if (ok) { s.names.push_back(nm); s.fields.push_back(std::move(v)); }
    }
    s.y.clear();
    if (ok && has_y) {
        s.y.resize(s.Ny);
        ok = std::fread(s.y.data(), 8, s.Ny, f) == (size_t)s.Ny;
    }
    std::fclose(f);
    if (!ok) err = "truncated snapshot " + path;
    return ok;
}

}  // namespace nse2d_host
