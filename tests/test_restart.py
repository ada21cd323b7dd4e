"""ParaView / restart files (frg_write_paraview_host, frg_read_restart_host)
against the reference's own writer and reader.

tests/golden/reference_paraview.npz (made by tests/golden/make_paraview_golden.py
from the reference itself) holds, for 3D hex cases, the state the reference's
writeParaview (src/output.cpp:103-391) wrote from, the file it wrote, and the
state its readRestartFile (src/solver.cpp:1420-1482, src/ele.cpp:1451-1880)
recovered from that file.  The host-side writer here must produce the same
bytes and the reader the same state and time.
"""
import os

import numpy as np
import pytest

from fr_learn_b200 import Mesh, box2d, box3d
from fr_learn_b200.solver import FrgError, read_restart_host, write_paraview_host

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_paraview.npz")
CASES = ("euler_p2", "euler_p3_cfl", "advection_p1")


def golden(name):
    z = np.load(GOLD)
    g = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}
    kw = dict(nDims=3, order=int(g["order"][0]), equation=int(g["equation"][0]))
    return g, kw


@pytest.mark.parametrize("name", CASES)
def test_writer_matches_reference_bytes(name, tmp_path):
    g, kw = golden(name)
    it = int(g["iter"][0])
    base = str(tmp_path / "sol")
    write_paraview_host(Mesh(3, g["xv"], None, None), g["U_spts"], float(g["time"][0]), it, base, **kw)
    with open(f"{base}_{it:09d}.vtu", "rb") as f:
        assert f.read() == g["vtu"].tobytes()


@pytest.mark.parametrize("name", CASES)
def test_reader_matches_reference_reader(name, tmp_path):
    g, kw = golden(name)
    it = int(g["iter"][0])
    base = str(tmp_path / "ref")
    with open(f"{base}_{it:09d}.vtu", "wb") as f:
        f.write(g["vtu"].tobytes())
    U, t = read_restart_host(g["xv"].shape[0], base, it, **kw)
    assert t == float(g["restart_time"][0])
    assert np.array_equal(U, g["restart_U_spts"])
    # 16 significant digits: the restart is within a few ulp of the written state
    assert np.abs(U - g["U_spts"]).max() <= 1e-14 * np.abs(g["U_spts"]).max()


def _state(nS, nE, nV, seed):
    rng = np.random.default_rng(seed)
    U = rng.uniform(0.5, 1.5, (nS, nE, nV))
    if nV > 1:
        U[..., -1] += 3.0  # positive pressure
    return U


@pytest.mark.parametrize("nDims,order,equation", [(2, 3, 1), (2, 5, 1), (2, 2, 0), (3, 4, 1)])
def test_round_trip(tmp_path, nDims, order, equation):
    mesh = box2d(4, 3, perturb=0.1, seed=2) if nDims == 2 else box3d(3, 3, 3, perturb=0.1, seed=3)
    nS, nV = (order + 1) ** nDims, (1 if equation == 0 else nDims + 2)
    U = _state(nS, mesh.nEles, nV, order)
    base = str(tmp_path / "rt")
    kw = dict(nDims=nDims, order=order, equation=equation)
    write_paraview_host(mesh, U, 1.25e-3, 42, base, **kw)
    U2, t = read_restart_host(mesh.nEles, base, 42, **kw)
    assert t == 1.25e-3
    assert np.abs(U2 - U).max() <= 1e-14 * np.abs(U).max()


def test_restart_at_another_order(tmp_path):
    """A P=2 file read by a P=4 solver: the inter-order Lagrange
    interpolation reproduces a field that is quadratic in each reference
    coordinate (ele::restart, src/ele.cpp:1506-1555, 1864-1873)."""
    mesh = box2d(3, 3)
    nE = mesh.nEles

    def field(P):
        x = np.polynomial.legendre.leggauss(P + 1)[0]  # the solution points, ascending
        X, Y = np.meshgrid(x, x)  # [j][i]: x fastest
        q = (1.0 + 0.3 * X - 0.2 * X * X) * (2.0 + 0.1 * Y + 0.4 * Y * Y)
        return np.repeat(q.ravel()[:, None, None], nE, axis=1)

    base = str(tmp_path / "ord")
    write_paraview_host(mesh, field(2), 0.5, 3, base, nDims=2, order=2, equation=0)
    U4, t = read_restart_host(nE, base, 3, nDims=2, order=4, equation=0)
    assert t == 0.5
    assert np.abs(U4 - field(4)).max() < 1e-14


def test_reader_errors(tmp_path):
    base = str(tmp_path / "none")
    with pytest.raises(FrgError) as ei:
        read_restart_host(4, base, 1, nDims=2, order=2)
    assert ei.value.code == 1
    mesh = box2d(3, 3)
    U = _state(9, mesh.nEles, 4, 0)
    write_paraview_host(mesh, U, 0.0, 1, base, nDims=2, order=2)
    path = f"{base}_{1:09d}.vtu"
    text = open(path).read().replace('Name="Pressure"', 'Name="Other"')
    open(path, "w").write(text)
    with pytest.raises(FrgError, match="missing"):
        read_restart_host(mesh.nEles, base, 1, nDims=2, order=2)


def test_short_file_fills_missing_elements(tmp_path, capfd):
    """A file with fewer pieces than the mesh has elements: like ele::restart
    (src/ele.cpp:1469-1478) the reader reports each missing element, sets
    its solution to 100 in every field and reads on; the elements the file
    holds are restored as usual."""
    base = str(tmp_path / "short")
    mesh = box2d(3, 3)
    U = _state(9, mesh.nEles, 4, 0)
    write_paraview_host(mesh, U, 0.5, 1, base, nDims=2, order=2)
    U2, t = read_restart_host(mesh.nEles + 2, base, 1, nDims=2, order=2)
    assert t == 0.5
    assert np.abs(U2[:, :mesh.nEles] - U).max() <= 1e-14 * np.abs(U).max()
    assert np.all(U2[:, mesh.nEles:] == 100.0)
    assert capfd.readouterr().out.count("Restart-file element doesn't exist!") == 2
