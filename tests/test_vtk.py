"""VTK output (WriteVTK, src/StokesVelocity.cc:773-993): the host writer of the C ABI
(ves3d_vtk_write_grid) fed with surfaces taken to the output order by the oracle, read back
and checked against the reference's layout; the pole weights against the oracle. CPU only."""
import ctypes
import os

import numpy as np
import pytest

from oracle import sh
from tests.helpers import rel_err, unit_sphere
from ves3d_b200 import _lib, vtk


def spheres(p, centres, radii):
    X = unit_sphere(p).reshape(3, -1)
    return np.concatenate([(r * X + np.asarray(c, float)[:, None]).reshape(-1) for c, r in zip(centres, radii)])


def to_order(X, p0, p1):
    """oracle: grid at p0 -> (grid at p1, poles) as WriteVTK upsamples (:780-784)."""
    S = sh.grid2shc(X, p0, p0)
    return sh.shc2grid(S, p0, p1), sh.shc2pole(S, p0)


def reference_polygons(p1, n_ves):
    """The reference's polygon loop (:843-875), restated."""
    con, off = [], []
    npt = 2 * p1 * (p1 + 1) + 2
    for k in range(n_ves):
        b = npt * k
        for j in range(2 * p1):
            j0, j1 = j, (j + 1) % (2 * p1)
            con += [b + 2 * p1 * (p1 + 1), b + j0, b + j1]
            off.append(len(con))
            con += [b + 2 * p1 * (p1 + 1) + 1, b + 2 * p1 * p1 + j0, b + 2 * p1 * p1 + j1]
            off.append(len(con))
        for i in range(p1):
            for j in range(2 * p1):
                j0, j1 = j, (j + 1) % (2 * p1)
                con += [b + 2 * p1 * i + j0, b + 2 * p1 * (i + 1) + j0, b + 2 * p1 * (i + 1) + j1, b + 2 * p1 * i + j1]
                off.append(len(con))
    return np.array(con, np.int32), np.array(off, np.int32)


def polygons(d):
    con, off = d["connectivity"], d["offsets"]
    start = np.concatenate([[0], off[:-1]])
    return [con[a:b] for a, b in zip(start, off)]


def test_pole_weights_match_the_closed_form_and_the_oracle():
    """The library's SHC2Pole table (recurrence of LegPoly) = sqrt(2 pi) times the normalised
    Legendre functions at the poles, (-+1)^n sqrt((2n+1)/2)."""
    for p in (2, 6, 12, 16, 32):
        qp = _lib.tables_export(p, 2 * p, "qp").reshape(2, p + 1)
        n = np.arange(p + 1)
        w = np.sqrt((2.0 * n + 1.0) / 2.0)
        assert rel_err(qp, np.stack([(-1.0) ** n * w, w])) < 1e-13
        # the oracle's SHC2Pole on unit m = 0 coefficients gives the same table
        S = np.zeros((p + 1, sh.ncoef(p)))
        S[n, n] = 1.0
        assert rel_err(qp.T.reshape(-1), sh.shc2pole(S, p)) < 1e-13


def sphere_mesh_volume_error(tmp_path, p0, p1, centres, radii):
    X1, Xp = to_order(spheres(p0, centres, radii), p0, p1)
    vtk.write_grid(X1, Xp, p1, str(tmp_path / "s"))
    d = vtk.read_vtp(str(tmp_path / "s_000000.vtp"))
    ng, npt = 2 * p1 * (p1 + 1), 2 * p1 * (p1 + 1) + 2
    P = d["points"]
    assert P.shape == (2 * npt, 3) and d["value"] is None
    for k, (c, r) in enumerate(zip(centres, radii)):
        Pk = P[k * npt:(k + 1) * npt]
        assert np.array_equal(Pk[:ng], X1.reshape(2, 3, ng)[k].T)  # grid copied as is
        assert np.array_equal(Pk[ng:], Xp.reshape(2, 3, 2)[k].T)
        assert np.allclose(np.linalg.norm(Pk - np.asarray(c), axis=1), r, atol=1e-12)
        # x = -1 pole is the south pole of this parametrisation, x = +1 the north pole
        assert np.allclose(Pk[ng], np.asarray(c) - [0, 0, r], atol=1e-12)
        assert np.allclose(Pk[ng + 1], np.asarray(c) + [0, 0, r], atol=1e-12)
    polys = polygons(d)
    assert len(polys) == 2 * (4 * p1 + 2 * p1 * p1)
    # The reference lists both pole fans in the same index order, so the fan at the x = +1
    # pole is wound against the rest of the mesh: each of its rim edges runs the same way as
    # the neighbouring quad's. Turned around, the mesh is closed and consistently oriented.
    rim = {}
    for poly in polys:
        for a, b in zip(poly, np.roll(poly, -1)):
            rim[(int(a), int(b))] = rim.get((int(a), int(b)), 0) + 1
    assert sum(n == 2 for n in rim.values()) == 2 * 2 * p1  # the x = +1 rims of both vesicles
    polys = [poly[::-1] if int(poly[0]) % npt == ng + 1 else poly for poly in polys]
    edges = {}
    for poly in polys:
        for a, b in zip(poly, np.roll(poly, -1)):
            edges[(int(a), int(b))] = edges.get((int(a), int(b)), 0) + 1
    assert all(n == 1 for n in edges.values())
    assert all((b, a) in edges for (a, b) in edges)
    # enclosed volume by the divergence theorem over fan triangles (quads on the grid)
    vols = np.zeros(2)
    for poly in polys:
        k = int(poly[0]) // npt
        for t in range(1, len(poly) - 1):
            vols[k] += np.linalg.det(P[[poly[0], poly[t], poly[t + 1]]] - np.asarray(centres[k])) / 6.0
    exact = 4.0 / 3.0 * np.pi * np.asarray(radii) ** 3
    assert np.all(np.sign(vols) == np.sign(vols[0]))
    return 1.0 - np.abs(vols) / exact


def test_sphere_mesh_is_closed_and_encloses_its_volume(tmp_path):
    """Points on the spheres, poles where they belong, a closed mesh, and the volume of the
    inscribed polyhedron below the sphere's, converging at second order in the spacing."""
    centres, radii = [(0, 0, 0), (4.0, 0.5, -1.0)], [1.0, 0.5]
    e12 = sphere_mesh_volume_error(tmp_path, 6, 12, centres, radii)
    e24 = sphere_mesh_volume_error(tmp_path, 6, 24, centres, radii)
    assert np.all((e12 > 0) & (e12 < 0.03)) and np.all((e24 > 0) & (e24 < 0.01))
    assert np.all(np.abs(e12 / e24 - 4.0) < 0.4)


def test_header_and_block_offsets_are_the_reference_layout(tmp_path):
    p1, nv = 2, 2
    ng = 2 * p1 * (p1 + 1)
    rng = np.random.default_rng(5)
    X1, Xp = rng.standard_normal(nv * 3 * ng), rng.standard_normal(nv * 6)
    V1, Vp = rng.standard_normal(nv * 3 * ng), rng.standard_normal(nv * 6)
    vtk.write_grid(X1, Xp, p1, str(tmp_path / "h"), V1, Vp)
    raw = open(tmp_path / "h_000000.vtp", "rb").read()
    npt = nv * (ng + 2)
    ncon, npoly = nv * (2 * p1 * 3 * 2 + p1 * 2 * p1 * 4), nv * (4 * p1 + 2 * p1 * p1)
    o_val = 4 + npt * 24
    o_con = o_val + 4 + npt * 24
    o_off = o_con + 4 + ncon * 4
    head = ('<?xml version="1.0"?>\n'
            '<VTKFile type="PolyData" version="0.1" byte_order="LittleEndian">\n'
            '  <PolyData>\n'
            f'    <Piece NumberOfPoints="{npt}" NumberOfVerts="0" NumberOfLines="0" NumberOfStrips="0" '
            f'NumberOfPolys="{npoly}">\n'
            '      <Points>\n'
            '        <DataArray type="Float64" NumberOfComponents="3" Name="Position" format="appended" offset="0" />\n'
            '      </Points>\n'
            '      <PointData>\n'
            f'        <DataArray type="Float64" NumberOfComponents="3" Name="value" format="appended" offset="{o_val}" />\n'
            '      </PointData>\n'
            '      <Polys>\n'
            f'        <DataArray type="Int32" Name="connectivity" format="appended" offset="{o_con}" />\n'
            f'        <DataArray type="Int32" Name="offsets" format="appended" offset="{o_off}" />\n'
            '      </Polys>\n'
            '    </Piece>\n'
            '  </PolyData>\n'
            '  <AppendedData encoding="raw">\n'
            '    _').encode()
    assert raw.startswith(head)
    body = raw[len(head):]
    tail = b'\n  </AppendedData>\n</VTKFile>\n'
    assert body.endswith(tail)
    assert len(body) == o_off + 4 + npoly * 4 + len(tail)
    sizes = [int(np.frombuffer(body, "<i4", 1, o)[0]) for o in (0, o_val, o_con, o_off)]
    assert sizes == [npt * 24, npt * 24, ncon * 4, npoly * 4]
    d = vtk.read_vtp(str(tmp_path / "h_000000.vtp"))
    Vg = V1.reshape(nv, 3, ng).transpose(0, 2, 1)
    Vq = Vp.reshape(nv, 3, 2).transpose(0, 2, 1)
    assert np.array_equal(d["value"], np.concatenate([Vg, Vq], axis=1).reshape(-1, 3))


@pytest.mark.parametrize("p1,nv", [(1, 1), (3, 2), (16, 3)])
def test_polygons_follow_the_reference_order(tmp_path, p1, nv):
    ng = 2 * p1 * (p1 + 1)
    vtk.write_grid(np.zeros(nv * 3 * ng), np.zeros(nv * 6), p1, str(tmp_path / "q"))
    d = vtk.read_vtp(str(tmp_path / "q_000000.vtp"))
    con, off = reference_polygons(p1, nv)
    assert np.array_equal(d["connectivity"], con)
    assert np.array_equal(d["offsets"], off)


def test_period_recentres_each_vesicle(tmp_path):
    p0, period = 6, 2.0
    shift = np.array([2.6 * period, -2.6 * period, 0.4 * period])  # C round(): 3, -3, 0
    centres = [(0.0, 0.0, 0.0), tuple(shift)]
    X1, Xp = to_order(spheres(p0, centres, [1.0, 1.0]), p0, p0)
    vtk.write_grid(X1, Xp, p0, str(tmp_path / "r"), period=period)
    P = vtk.read_vtp(str(tmp_path / "r_000000.vtp"))["points"]
    npt = 2 * p0 * (p0 + 1) + 2
    assert np.allclose(P[:npt].mean(axis=0), 0.0, atol=1e-12)
    assert np.allclose(P[npt:].mean(axis=0), shift - period * np.array([3.0, -3.0, 0.0]), atol=1e-12)
    # period 0 leaves the points alone
    vtk.write_grid(X1, Xp, p0, str(tmp_path / "r0"))
    P0 = vtk.read_vtp(str(tmp_path / "r0_000000.vtp"))["points"]
    assert np.allclose(P0[npt:].mean(axis=0), shift, atol=1e-12)


def test_index_file_lists_every_rank_and_only_rank_0_writes_it(tmp_path):
    p1 = 2
    X1, Xp = np.zeros(3 * 2 * p1 * (p1 + 1)), np.zeros(6)
    base = str(tmp_path / "run" / "frame")
    os.makedirs(tmp_path / "run")
    vtk.write_grid(X1, Xp, p1, base, rank=1, n_ranks=3)
    assert os.path.exists(base + "_000001.vtp") and not os.path.exists(base + ".pvtp")
    vtk.write_grid(X1, Xp, p1, base, X1, Xp, rank=0, n_ranks=3)
    txt = open(base + ".pvtp").read()
    assert vtk.read_pvtp(base + ".pvtp") == ["frame_000000.vtp", "frame_000001.vtp", "frame_000002.vtp"]
    assert txt.startswith('<?xml version="1.0"?>\n<VTKFile type="PPolyData">\n  <PPolyData GhostLevel="0">\n')
    assert '<PDataArray type="Float64" NumberOfComponents="3" Name="value"/>' in txt
    vtk.write_grid(X1, Xp, p1, base, rank=0, n_ranks=1)  # no field: no PPointData
    assert "PPointData" not in open(base + ".pvtp").read()


def test_empty_suspension_writes_an_empty_piece(tmp_path):
    vtk.write_grid(np.zeros(0), np.zeros(0), 4, str(tmp_path / "e"))
    d = vtk.read_vtp(str(tmp_path / "e_000000.vtp"))
    assert d["points"].shape == (0, 3) and d["connectivity"].size == 0 and d["offsets"].size == 0


def test_errors(tmp_path):
    L = _lib.lib()
    z = np.zeros(3 * 12 + 6)
    st = L.ves3d_vtk_write_grid(z.ctypes.data, z.ctypes.data, None, None, 1, 2,
                                str(tmp_path / "no_such_dir" / "x").encode(), 0.0, 0, 1)
    assert st == 7 and b"cannot open" in L.ves3d_last_error()
    with pytest.raises(RuntimeError):
        vtk.write_grid(z[:36], z[36:], 2, str(tmp_path / "no_such_dir" / "x"))
    f = str(tmp_path / "x").encode()
    assert L.ves3d_vtk_write_grid(z.ctypes.data, z.ctypes.data, None, None, -1, 2, f, 0.0, 0, 1) == 1
    assert L.ves3d_vtk_write_grid(None, None, None, None, 1, 2, f, 0.0, 0, 1) == 1
    assert L.ves3d_vtk_write_grid(z.ctypes.data, z.ctypes.data, z.ctypes.data, None, 1, 2, f, 0.0, 0, 1) == 1
    assert L.ves3d_vtk_write_grid(z.ctypes.data, z.ctypes.data, None, None, 1, 0, f, 0.0, 0, 1) == 1
    assert L.ves3d_vtk_write_grid(z.ctypes.data, z.ctypes.data, None, None, 1, 2, f, 0.0, 2, 2) == 1
    assert L.ves3d_vtk_write_grid(z.ctypes.data, z.ctypes.data, None, None, 1, 2, None, 0.0, 0, 1) == 1
    assert L.ves3d_vtk_write_grid(z.ctypes.data, z.ctypes.data, None, None, 1, 2, f, float("nan"), 0, 1) == 1
    assert L.ves3d_vtk_write(None, None, 1, 6, 12, f, 0.0, 0, 1, 0) == 1
    assert L.ves3d_vtk_write(z.ctypes.data, None, 1, 0, 12, f, 0.0, 0, 1, 0) == 1
    assert L.ves3d_vtk_write(z.ctypes.data, None, 1, 6, 12, f, 0.0, -1, 1, 0) == 1
    assert L.ves3d_sht_pole(None, 1, 6, None, None) == 1
    assert L.ves3d_sht_pole(z.ctypes.data, 1, 0, z.ctypes.data, None) == 1
    with pytest.raises(ValueError):
        vtk.write_grid(z[:35], z[36:], 2, str(tmp_path / "x"))
    with pytest.raises(ValueError):
        vtk.WriteVTK(np.zeros(10), 6, 12, str(tmp_path / "x"))
    assert not os.path.exists(tmp_path / "x_000000.vtp")


def test_write_without_a_gpu_is_an_error_not_a_crash(tmp_path):
    from tests.conftest import cuda_available
    if cuda_available():
        pytest.skip("GPU present")
    p = 6
    X = spheres(p, [(0, 0, 0)], [1.0])
    st = _lib.lib().ves3d_vtk_write(X.ctypes.data, None, 1, p, 2 * p, str(tmp_path / "g").encode(), 0.0, 0, 1, 0)
    assert st in (2, 5)
    assert not os.path.exists(tmp_path / "g_000000.vtp")
    assert ctypes.string_at(_lib.lib().ves3d_last_error())


def test_rank_without_size_is_rejected():
    """An explicit rank needs its communicator size and the other way round (a guessed
    size would write the index from the wrong process or collide piece names)."""
    with pytest.raises(ValueError):
        vtk._rank_size(1, None)
    with pytest.raises(ValueError):
        vtk._rank_size(None, 2)
    assert vtk._rank_size(1, 2) == (1, 2)
