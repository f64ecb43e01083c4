#include "snapshot.h"

#include <cstdint>
#include <cstdio>
#include <cstring>

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

bool read_snapshot(const std::string& path, Snapshot& s, std::string& err) {
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
