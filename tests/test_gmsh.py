"""The Gmsh v2 reader (frg_read_gmsh: geo::readGmsh, src/geo.cpp:448-769, and
the boundary matching of geo::processConn3D, src/geo.cpp:169-193).  CPU only.

3D: the meshes of the reference-pinned cases (tests/golden/reference_golden.npz)
are written as Gmsh files the way they were written for the reference
(tests/refcase.py write_gmsh, physical names = condition names); read back,
they give the same elements, corners and boundary conditions, and the set-up
built from them has the reference's own face table, solution-point
positions and Jacobians.  2D: a 9-node quad channel written as a Gmsh file
(type-10 quads, type-8 boundary edges) reads back to the same arrays.
"""
import os

import numpy as np
import pytest

from conftest import relerr

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "reference_golden.npz")
CASES = ["euler_p2_char_fixeddt", "euler_p2_charslip_cfl", "ns_p3_walls"]


def _bounds(names):
    return {n: n for n in names} | {"fluid": "fluid"}


@pytest.mark.parametrize("name", CASES)
def test_gmsh_3d_matches_reference_setup(tmp_path, name):
    import refcase
    from fr_learn_b200 import read_gmsh
    from fr_learn_b200.mesh import Mesh
    from fr_learn_b200.solver import inspect_geometry

    g = np.load(GOLDEN)
    pre = f"case/{name}/"
    xv, c2v = g[pre + "xv"], g[pre + "c2v"]
    verts = np.zeros((int(c2v.max()) + 1, 3))
    verts[c2v.ravel()] = xv.reshape(-1, 3)
    mesh = Mesh(3, xv, c2v, g[pre + "bc"], verts=verts)
    path = str(tmp_path / "m.msh")
    names = refcase.write_gmsh(mesh, path)
    r = read_gmsh(path, _bounds(names))
    assert r.nDims == 3 and r.nEles == mesh.nEles and r.nNodes == 8
    assert np.array_equal(r.xv, mesh.xv)
    assert np.array_equal(r.bc, mesh.bc)
    order = int(g[pre + "setup"][0])
    fa = inspect_geometry(r, "faces", order=order)
    assert sorted(map(tuple, fa.tolist())) == sorted(map(tuple, g[pre + "faces"].tolist()))
    pos = inspect_geometry(r, "pos_spts", order=order)
    assert relerr(pos, g[pre + "pos_spts"]) < 1e-14
    assert relerr(inspect_geometry(r, "detJac_spts", order=order), g[pre + "detJac_spts"]) < 1e-14


def _write_gmsh_2d(mesh, path, names):
    """Gmsh v2 file of 9-node quads with 3-node boundary edges (corners of
    each edge first, as Gmsh orders them)."""
    from fr_learn_b200.mesh import BC

    inv = {v: k for k, v in BC.items()}
    # unique nodes by coordinates
    key, first = {}, []
    ids = np.zeros(mesh.xv.shape[:2], np.int64)
    for e in range(mesh.nEles):
        for n in range(9):
            k = tuple(np.round(mesh.xv[e, n], 12))
            if k not in key:
                key[k] = len(first)
                first.append(mesh.xv[e, n])
            ids[e, n] = key[k]
    coords = np.array(first)
    phys = {b: i + 1 for i, b in enumerate(sorted({int(b) for b in mesh.bc.ravel() if b >= 0}))}
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(phys) + 1)]
    for b, i in phys.items():
        lines.append(f'1 {i} "{names[inv[b]]}"')
    lines += ['2 99 "Domain"', "$EndPhysicalNames", "$Nodes", str(len(coords))]
    lines += [f"{i + 1} {float(c[0])!r} {float(c[1])!r} 0" for i, c in enumerate(coords)]
    lines += ["$EndNodes", "$Elements"]
    els = []
    edge = ((0, 1, 4), (1, 2, 5), (2, 3, 6), (3, 0, 7))
    for e in range(mesh.nEles):
        for f in range(4):
            b = int(mesh.bc[e, f])
            if b >= 0:
                els.append(f"8 2 {phys[b]} {phys[b]} " + " ".join(str(ids[e, k] + 1) for k in edge[f]))
    for e in range(mesh.nEles):
        els.append("10 2 99 99 " + " ".join(str(ids[e, n] + 1) for n in range(9)))
    lines.append(str(len(els)))
    lines += [f"{i + 1} {s}" for i, s in enumerate(els)]
    lines.append("$EndElements")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def test_gmsh_2d_quadratic_quads_round_trip(tmp_path):
    from fr_learn_b200 import bump2d, read_gmsh

    mesh = bump2d(8, 3)
    names = {"char": "Farfield", "slip_wall": "Wall"}
    path = str(tmp_path / "bump.msh")
    _write_gmsh_2d(mesh, path, names)
    r = read_gmsh(path, "farfield char; WALL slip_wall; domain fluid")
    assert r.nDims == 2 and r.nNodes == 9 and r.nEles == mesh.nEles
    assert np.array_equal(r.xv, mesh.xv)
    assert np.array_equal(r.bc, mesh.bc)


def test_gmsh_errors(tmp_path):
    from fr_learn_b200 import FrgError, bump2d, read_gmsh

    mesh = bump2d(4, 2)
    path = str(tmp_path / "b.msh")
    _write_gmsh_2d(mesh, path, {"char": "Farfield", "slip_wall": "Wall"})
    with pytest.raises(FrgError, match="Unrecognized mesh boundary"):
        read_gmsh(path, "farfield char; domain fluid")
    with pytest.raises(FrgError, match="Unrecognized boundary condition"):
        read_gmsh(path, "farfield char; wall nowall; domain fluid")
    with pytest.raises(FrgError, match="Unable to open"):
        read_gmsh(str(tmp_path / "none.msh"), "domain fluid")
