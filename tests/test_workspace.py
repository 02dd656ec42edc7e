"""Workspace files (qesb_workspace_write / _read): NetCDF classic with the
reference's workspace variables (src/winds/WINDSOutputWorkspace.cpp:40-154).
Checked against scipy's own NetCDF classic reader and writer, an independent
implementation of the format."""
import numpy as np
import pytest

import qesb

scipy_io = pytest.importorskip("scipy.io")


def _city():
    d = qesb.Domain(30, 26, 12, 2.0, 2.5, 1.0, qesb.city_dz(12, 1.0, 1.04))
    c = qesb.city_random(d, 21, 4, fp=(6, 12), h=(4, 10))
    w = qesb.city_build(d, c.buildings, c.inflow)
    rng = np.random.default_rng(3)
    for name in ("u", "v", "w"):
        setattr(w, name, rng.standard_normal(d.numFaceCentered()).astype(np.float32))
    return d, w


def test_written_file_reads_back_in_scipy(tmp_path):
    d, w = _city()
    path = str(tmp_path / "ws.nc")
    qesb.workspace_write(path, w, t=12.5)
    with open(path, "rb") as fh:
        assert fh.read(4) == b"CDF\x02"
    nz, ny, nx = d.face_shape()
    with scipy_io.netcdf_file(path, "r", mmap=False) as f:
        assert f.dimensions["t"] is None and f.dimensions["x_face"] == nx and f.dimensions["z"] == nz - 1
        assert float(f.variables["t"].data[0]) == 12.5
        for name in ("u", "v", "w", "u0", "v0", "w0"):
            var = f.variables[name]
            assert var.dimensions == ("t", "z_face", "y_face", "x_face")
            np.testing.assert_array_equal(var.data[0].ravel(), getattr(w, name))
            assert var.units == b"m s-1"
        for name in ("e", "f", "g", "h", "m", "n"):
            assert f.variables[name].dimensions == ("t", "z", "y", "x")
            np.testing.assert_array_equal(f.variables[name].data[0].ravel(), getattr(w, name))
        assert f.variables["icellflag"].data.dtype.kind == "i"
        np.testing.assert_array_equal(f.variables["icellflag"].data[0].ravel(), w.icellflag)
        assert f.variables["icellflag"].long_name == b"icell flag value"
        np.testing.assert_array_equal(f.variables["dz_array"].data, d.dz_array)
        # coordinates as WINDSOutputWorkspace.cpp:50-88 sets them
        x = f.variables["x"].data
        np.testing.assert_allclose(x, (np.arange(nx - 1) + 0.5) * 2.0)
        np.testing.assert_allclose(f.variables["x_face"].data, np.concatenate([[x[0] - 2.0], x]))
        y = f.variables["y"].data
        np.testing.assert_allclose(f.variables["y_face"].data, np.concatenate([[y[0] - 2.5], y + 2.5]))
        np.testing.assert_array_equal(f.variables["z_face"].data, d.z_face)
        np.testing.assert_array_equal(f.variables["z"].data, d.z)


def test_round_trip(tmp_path):
    d, w = _city()
    path = str(tmp_path / "ws.nc")
    qesb.workspace_write(path, w)
    r = qesb.workspace_read(path)
    assert r.domain.base == d.base and r.domain.dx() == d.dx() and r.domain.dy() == d.dy()
    np.testing.assert_array_equal(r.domain.dz_array, d.dz_array)
    for name in ("icellflag", "e", "f", "g", "h", "m", "n", "u0", "v0", "w0", "u", "v", "w"):
        np.testing.assert_array_equal(getattr(r, name), getattr(w, name))


@pytest.mark.parametrize("version", [1, 2])
def test_reads_files_written_by_scipy(tmp_path, version):
    """Classic files from another writer, with other numeric types (double
    winds, short flags) and extra variables, in either header version."""
    d, w = _city()
    nz, ny, nx = d.face_shape()
    path = str(tmp_path / "other.nc")
    with scipy_io.netcdf_file(path, "w", version=version) as f:
        f.createDimension("t", None)
        for name, n in (("x_face", nx), ("y_face", ny), ("z_face", nz), ("x", nx - 1), ("y", ny - 1),
                        ("z", nz - 1)):
            f.createDimension(name, n)
        f.createVariable("x", "f4", ("x",))[:] = (np.arange(nx - 1) + 0.5) * d.dx()
        f.createVariable("y", "f4", ("y",))[:] = (np.arange(ny - 1) + 0.5) * d.dy()
        f.createVariable("dz_array", "f4", ("z",))[:] = d.dz_array
        f.createVariable("terrain", "f4", ("y", "x"))[:] = 0.0
        for name in ("u", "v", "w", "u0", "v0", "w0"):
            v = f.createVariable(name, "f8", ("t", "z_face", "y_face", "x_face"))
            v[0] = getattr(w, name).reshape(nz, ny, nx).astype(np.float64)
            v.units = "m s-1"
        f.createVariable("icellflag", "i2", ("t", "z", "y", "x"))[0] = w.icellflag.reshape(d.cell_shape())
        for name in ("e", "f", "g", "h", "m", "n"):
            f.createVariable(name, "f4", ("t", "z", "y", "x"))[0] = getattr(w, name).reshape(d.cell_shape())
    r = qesb.workspace_read(path)
    assert r.domain.base == d.base
    for name in ("icellflag", "e", "f", "g", "h", "m", "n", "u0", "v0", "w0", "u", "v", "w"):
        np.testing.assert_array_equal(getattr(r, name), getattr(w, name))


def test_rejects_netcdf4_and_wrong_grids(tmp_path):
    h5 = tmp_path / "nc4.nc"
    h5.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(64))
    with pytest.raises(qesb.QesbError, match="nccopy"):
        qesb.workspace_read(str(h5))
    d, w = _city()
    path = str(tmp_path / "ws.nc")
    qesb.workspace_write(path, w)
    e = np.empty(10, np.float32)
    st = qesb.lib().qesb_workspace_read(path.encode(), 31, 26, 12, None, None, e.ctypes.data, *[None] * 11)
    assert st != 0 and "grid" in qesb.lib().qesb_last_error().decode()


def test_large_header_and_truncated_files(tmp_path):
    """A header longer than the reader's first 64 KB prefix (many variables
    with long attributes) is read in full; a file cut inside its header is
    refused."""
    d, w = _city()
    nz, ny, nx = d.face_shape()
    path = str(tmp_path / "big_header.nc")
    with scipy_io.netcdf_file(path, "w", version=2) as f:
        f.createDimension("t", None)
        for name, n in (("x_face", nx), ("y_face", ny), ("z_face", nz), ("x", nx - 1), ("y", ny - 1),
                        ("z", nz - 1)):
            f.createDimension(name, n)
        for q in range(400):  # ~400 x 220 bytes of header before the fields
            v = f.createVariable(f"extra_{q:03d}", "f4", ("z",))
            v.long_name = "padding attribute " + "x" * 180
            v[:] = q
        f.createVariable("x", "f4", ("x",))[:] = (np.arange(nx - 1) + 0.5) * d.dx()
        f.createVariable("y", "f4", ("y",))[:] = (np.arange(ny - 1) + 0.5) * d.dy()
        f.createVariable("dz_array", "f4", ("z",))[:] = d.dz_array
        for name in ("u", "v", "w", "u0", "v0", "w0"):
            f.createVariable(name, "f4", ("t", "z_face", "y_face", "x_face"))[0] = \
                getattr(w, name).reshape(nz, ny, nx)
        f.createVariable("icellflag", "i4", ("t", "z", "y", "x"))[0] = w.icellflag.reshape(d.cell_shape())
        for name in ("e", "f", "g", "h", "m", "n"):
            f.createVariable(name, "f4", ("t", "z", "y", "x"))[0] = getattr(w, name).reshape(d.cell_shape())
    r = qesb.workspace_read(path)
    for name in ("icellflag", "e", "n", "u0", "w"):
        np.testing.assert_array_equal(getattr(r, name), getattr(w, name))
    cut = tmp_path / "cut.nc"
    cut.write_bytes(open(path, "rb").read()[:70000])
    with pytest.raises(qesb.QesbError, match="truncated"):
        qesb.workspace_read(str(cut))
