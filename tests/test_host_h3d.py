"""Hydro3D restart exchange and Ghia post-processing (no GPU).

Pinned to the reference's own code: tests/golden/golden_tecbin_8.npz holds
the tecbin file the reference's exporter (tests/h3d_bridge.py) wrote for a
freshly initialised 8^3 cavity, the real cells it wrote it from, and what
the reference's reader returns for it (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from helpers import golden


@pytest.fixture(scope="module")
def g():
    return golden("tecbin_8")


def _h3d_fields(g):
    from warpflow import h3d
    bnd = dict((str(k), str(v)) for k, v in g["bnd"])
    n = int(g["n"])
    out = {name: h3d.fill_ghosts(g["real_" + name], name, bnd, h3d.PL_H3D, float(g["ulid"]))
           for name in ("u", "v", "w", "p")}
    out["vis"] = np.full_like(out["u"], float(g["rey"]))
    return out, n


def test_writer_matches_reference_bytes(g, tmp_path):
    from warpflow import h3d
    fields, n = _h3d_fields(g)
    path = str(tmp_path / "tecbin0000.bin")
    h3d.write_tecbin(path, fields, n, float(g["dx"]))
    np.testing.assert_array_equal(np.fromfile(path, np.uint8), g["tecbin"])


def test_reader_matches_reference_reader(g, tmp_path):
    from warpflow import h3d
    path = str(tmp_path / "ref.bin")
    g["tecbin"].tofile(path)
    n = int(g["n"])
    for raw, tag in ((False, "core_"), (True, "raw_")):
        got = h3d.read_tecbin(path, n, raw=raw)
        for name in ("u", "v", "w", "p", "vis"):
            np.testing.assert_array_equal(got[name], g[tag + name], err_msg=tag + name)
    # the real cells are the fields the reference exported
    core = h3d.read_tecbin(path, n)
    for name in ("u", "v", "w", "p"):
        np.testing.assert_array_equal(core[name], g["real_" + name])


def test_round_trip_and_corrupt_files(tmp_path):
    from warpflow import h3d
    n, pl = 6, h3d.PL_H3D
    rng = np.random.default_rng(11)
    fields = {k: rng.standard_normal((n + 2 * pl,) * 3) for k in ("u", "v", "w", "p", "vis")}
    path = str(tmp_path / "t.bin")
    h3d.write_tecbin(path, fields, n, 0.1)
    got = h3d.read_tecbin(path, n, raw=True)
    for k in fields:
        np.testing.assert_array_equal(got[k], fields[k])
    with pytest.raises(ValueError, match="expected"):
        h3d.read_tecbin(path, n + 2)
    data = np.fromfile(path, np.uint8)
    data[:-100].tofile(path)
    with pytest.raises(ValueError, match="truncated"):
        h3d.read_tecbin(path, n)


def test_final_ctime_line_matches_reference(g, tmp_path):
    line = "       0%18.12f%18.12f%18.12f\n" % (0.0, 0.0, 1.0)
    assert str(g["final_ctime"]) == line


def test_compare_pairs_planes(tmp_path):
    """A Hydro3D dump whose plane s holds this package's index s - 1 agrees
    exactly; pressure is compared demeaned."""
    from warpflow import h3d
    n, pl = 8, h3d.PL_H3D
    rng = np.random.default_rng(3)
    snap = {k: rng.standard_normal((n + 6,) * 3) for k in ("u", "v", "w", "p")}
    fields = {}
    for k in snap:
        a = np.zeros((n + 2 * pl,) * 3)
        a[1:n + 7, 1:n + 7, 1:n + 7] = snap[k]     # file plane s = array index s - 1
        fields[k] = a
    fields["p"] = fields["p"] + 5.0          # a constant offset in pressure only
    fields["vis"] = np.zeros_like(fields["u"])
    os.makedirs(tmp_path / "h3d")
    os.makedirs(tmp_path / "snap")
    h3d.write_tecbin(str(tmp_path / "h3d" / "h3d_it025.bin"), fields, n, 1.0 / n)
    np.savez(str(tmp_path / "snap" / "snap_000025_r000.npz"), **snap)
    out = h3d.compare(str(tmp_path / "h3d"), str(tmp_path / "snap"), n=n, step=25, upto=25)
    assert list(out) == [25]
    for k, (dmax, rms) in out[25].items():
        assert dmax <= 1e-12, (k, dmax)


def test_centreline_profiles_and_ghia_rms(tmp_path):
    from warpflow import h3d
    n = 8
    idx = np.arange(n + 6)
    u = idx[:, None, None] * 10000.0 + idx[None, :, None] * 100.0 + idx[None, None, :]
    w = -u
    zc, up, xc, wp = h3d.centreline_profiles(u, w)
    np.testing.assert_allclose(zc, (np.arange(n) + 0.5) / n)
    # u at x face n/2 (full n/2+2), y centre n/2 (full n/2+3), all z centres
    np.testing.assert_array_equal(up, u[6, 7, 3:3 + n])
    np.testing.assert_array_equal(wp, w[3:3 + n, 7, 6])
    ghia = (zc, up.copy())
    assert h3d.ghia_rms((zc, up, xc, wp), ghia, (xc, wp.copy())) == (0.0, 0.0)
    path = str(tmp_path / "c.csv")
    h3d.write_centreline_csv(path, (zc, up, xc, wp))
    rows = open(path).read().splitlines()
    assert rows[0] == "z,u_centerline,x,w_centerline" and len(rows) == n + 1
