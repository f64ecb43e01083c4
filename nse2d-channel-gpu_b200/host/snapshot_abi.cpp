// C ABI of the snapshot files (include/nse2d.h, group 5): the reference's HDF5 layout
// (src/io.cu:183-259) and the flat "bin" layout, through host/snapshot.cpp and host/h5lite.cpp.
// Host code only: these entry points touch no GPU. Written for this project.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nse2d.h"
#include "snapshot.h"

namespace nse2d {
void set_error(const char* fmt, ...);
}

using nse2d_host::Snapshot;

extern "C" {

int nse2d_snapshot_write(const char* path, int format, const nse2d_snapshot_meta* m, int nfields,
                         const char* const* names, const double* const* fields) {
    if (!path || !m || nfields < 0 || nfields > 8 || (nfields > 0 && (!names || !fields))) {
        nse2d::set_error("nse2d_snapshot_write: bad arguments");
        return -1;
    }
    if (m->Nx < 1 || m->Ny < 2) { nse2d::set_error("nse2d_snapshot_write: bad grid %d x %d", m->Nx, m->Ny); return -1; }
    Snapshot s;
    s.Nx = m->Nx; s.Ny = m->Ny; s.t = m->t; s.Lx = m->Lx; s.h = m->h; s.nu = m->nu; s.beta = m->beta;
    s.tanh = m->stretch_tanh != 0;
    const size_t N = (size_t)m->Nx * m->Ny;
    for (int q = 0; q < nfields; ++q) {
        if (!names[q] || !fields[q]) { nse2d::set_error("nse2d_snapshot_write: null field %d", q); return -1; }
        s.names.push_back(names[q]);
        s.fields.emplace_back(fields[q], fields[q] + N);
    }
    if (m->y) s.y.assign(m->y, m->y + m->Ny);
    std::string err;
    const bool ok = (format == 0) ? nse2d_host::write_snapshot_h5(path, s, err)
                  : (format == 1) ? nse2d_host::write_snapshot(path, s, err)
                                  : (err = "unknown snapshot format", false);
    if (!ok) { nse2d::set_error("nse2d_snapshot_write: %s", err.c_str()); return -1; }
    return 0;
}

int nse2d_snapshot_read(const char* path, nse2d_snapshot_meta* m, const char* name, double* out) {
    if (!path) { nse2d::set_error("nse2d_snapshot_read: null path"); return -1; }
    Snapshot s;
    std::string err;
    if (!nse2d_host::read_snapshot(path, s, err)) { nse2d::set_error("nse2d_snapshot_read: %s", err.c_str()); return -1; }
    if (m) {
        m->Nx = s.Nx; m->Ny = s.Ny; m->t = s.t; m->Lx = s.Lx; m->h = s.h; m->nu = s.nu; m->beta = s.beta;
        m->stretch_tanh = s.tanh ? 1 : 0;
        m->y = nullptr;
        m->fields = 0;
        for (size_t q = 0; q < s.names.size() && q < 8; ++q) {
            if (s.names[q] == "omega") m->fields |= 1;
            else if (s.names[q] == "psi") m->fields |= 2;
            else if (s.names[q] == "u") m->fields |= 4;
            else if (s.names[q] == "v") m->fields |= 8;
        }
        if (!s.y.empty()) m->fields |= 16;
    }
    if (name && out) {
        if (std::strcmp(name, "y") == 0) {
            if (s.y.empty()) { nse2d::set_error("nse2d_snapshot_read: %s has no y", path); return -1; }
            std::memcpy(out, s.y.data(), s.y.size() * sizeof(double));
            return 0;
        }
        const std::vector<double>* f = s.field(name);
        if (!f) { nse2d::set_error("nse2d_snapshot_read: %s has no field %s", path, name); return -1; }
        std::memcpy(out, f->data(), f->size() * sizeof(double));
    }
    return 0;
}

}  // extern "C"
