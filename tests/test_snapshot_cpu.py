"""Snapshot files on the CPU (no GPU): the reference's HDF5 layout (src/io.cu:183-259) as written by
this library (nse2d_snapshot_write, host/h5lite.cpp, no libhdf5), checked with an independent
reader (tests/h5read.py, written from the HDF5 File Format Specification) and byte by byte against
the structures libhdf5 writes with its default properties; then read back by the library
(nse2d_snapshot_read), in both formats.

The image has no libhdf5 or h5py, so the files cannot be opened with them here; the layout is the
earliest-format one (superblock 0, symbol-table root group, version-1 object headers, contiguous
datasets) that every HDF5 reader supports.
"""
import os

import numpy as np
import pytest

from h5read import SIG, UNDEF, H5File


@pytest.fixture()
def fields():
    rng = np.random.default_rng(7)
    Nx, Ny = 16, 9
    y = np.tanh(2.0 * np.linspace(-1, 1, Ny)) / np.tanh(2.0)
    return dict(omega=rng.standard_normal((Ny, Nx)), psi=rng.standard_normal((Ny, Nx)),
                u=rng.standard_normal((Ny, Nx)), v=rng.standard_normal((Ny, Nx))), y


META = dict(t=0.35, Lx=2 * np.pi, h=1.0, nu=2e-4)


def test_hdf5_layout_and_values(nse, tmp_path, fields):
    f, y = fields
    p = tmp_path / "snap_t0.350000.h5"
    nse.write_snapshot(p, f, beta=2.0, y=y, **META)
    h = H5File(str(p))
    sb = h.structures["superblock"]
    # superblock version 0 (as libhdf5 writes with default properties), 8-byte offsets and lengths
    assert open(p, "rb").read(8) == SIG
    assert (sb["version"], sb["freespace_version"], sb["root_entry_version"], sb["shared_header_version"]) == (0, 0, 0, 0)
    assert (sb["leaf_k"], sb["internal_k"], sb["flags"]) == (4, 16, 0)
    assert sb["base"] == 0 and sb["freespace"] == UNDEF and sb["driver"] == UNDEF
    assert sb["eof"] == os.path.getsize(p)
    assert sb["root"]["cache_type"] == 1
    # the root group: one B-tree leaf whose child is one symbol table node, names in a local heap
    bt = h.structures["btree_nodes"]
    assert len(bt) == 1 and bt[0]["type"] == 0 and bt[0]["level"] == 0 and bt[0]["entries"] == 1
    assert bt[0]["left"] == UNDEF and bt[0]["right"] == UNDEF
    sn = h.structures["symbol_nodes"]
    names = [e["name"] for e in sn[0]["entries"]]
    assert sn[0]["version"] == 1 and names == sorted(names) == ["omega", "psi", "u", "v", "y"]
    assert bt[0]["keys"][0] == 0 and h.heap_name(bt[0]["keys"][1]) == names[-1]
    heap = h.structures["local_heap"]
    assert heap["version"] == 0 and heap["free_list"] == 1 and heap["data_size"] % 8 == 0
    # datasets: [Ny, Nx] little-endian float64, contiguous; y [1, Ny] (src/io.cu:236)
    for k in ("omega", "psi", "u", "v"):
        ds = h.dataset(k)
        assert ds.dims == [9, 16] and ds.dtype["cls"] == "float" and ds.dtype["size"] == 8
        assert ds.dtype["sign_bit"] == 63 and ds.dtype["props"] == (0, 64, 52, 11, 0, 52, 1023)
        assert np.array_equal(h.read(k), f[k])
    assert h.dataset("y").dims == [1, 9] and np.array_equal(h.read("y").ravel(), y)
    # root attributes (src/io.cu:240-255): Nx, Ny 32-bit signed integers, the rest float64
    a, types = h.attrs, h.structures["attr_types"]
    assert set(a) == {"beta", "stretch_code", "t", "Nx", "Ny", "Lx", "Ly", "h", "dx", "dy", "nu"}
    assert types["Nx"]["cls"] == "int" and types["Nx"]["size"] == 4 and types["Nx"]["signed"]
    assert all(types[k]["cls"] == "float" and types[k]["size"] == 8 for k in a if k not in ("Nx", "Ny"))
    assert all(types[k]["space"]["rank"] == 0 for k in a)
    assert (a["Nx"], a["Ny"]) == (16, 9)
    assert a["t"] == 0.35 and a["Lx"] == 2 * np.pi and a["Ly"] == 2.0 and a["h"] == 1.0 and a["nu"] == 2e-4
    assert a["dx"] == 2 * np.pi / 16 and a["dy"] == 2.0 / 8 and a["beta"] == 2.0 and a["stretch_code"] == 1.0


def test_uniform_grid_has_no_y(nse, tmp_path, fields):
    f, _ = fields
    p = tmp_path / "u.h5"
    nse.write_snapshot(p, {"omega": f["omega"]}, **META)
    h = H5File(str(p))
    assert list(h.links) == ["omega"]
    assert "beta" not in h.attrs and "stretch_code" not in h.attrs


@pytest.mark.parametrize("fmt", ["h5", "bin"])
def test_library_reads_back(nse, tmp_path, fields, fmt):
    f, y = fields
    p = tmp_path / f"s.{fmt}"
    nse.write_snapshot(p, {"omega": f["omega"], "psi": f["psi"]}, beta=2.0, y=y, fmt=fmt, **META)
    meta, got = nse.read_snapshot(p)
    assert (meta["Nx"], meta["Ny"], meta["t"], meta["Lx"], meta["h"], meta["nu"]) == (16, 9, 0.35, 2 * np.pi, 1.0, 2e-4)
    assert meta["stretch_tanh"] == 1 and meta["beta"] == 2.0
    assert sorted(got) == ["omega", "psi", "y"]
    assert np.array_equal(got["omega"], f["omega"]) and np.array_equal(got["psi"], f["psi"])
    assert np.array_equal(got["y"], y)


def test_reader_rejects_bad_files(nse, tmp_path, fields):
    f, _ = fields
    p = tmp_path / "a.h5"
    nse.write_snapshot(p, {"omega": f["omega"]}, **META)
    data = open(p, "rb").read()
    cut = tmp_path / "cut.h5"
    open(cut, "wb").write(data[:len(data) - 200])          # the data block runs past the end
    with pytest.raises(nse.Nse2dError, match="beyond the end|does not have"):
        nse.read_snapshot(cut)
    junk = tmp_path / "junk.h5"
    open(junk, "wb").write(b"not a snapshot" * 10)
    with pytest.raises(nse.Nse2dError):
        nse.read_snapshot(junk)
