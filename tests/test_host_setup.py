"""Host-side logic of the product, on CPU: the C ABI library loads and exports
every entry point include/frgpu.h declares; its set-up (metrics, normals,
face pairing incl. periodic and 3D relRot) equals the oracle's; mesh
generators; error paths that need no device."""
import os
import re

import numpy as np
import pytest

from conftest import relerr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "frgpu.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(frg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from fr_learn_b200.solver import lib

    L = lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_error_without_device():
    from fr_learn_b200.solver import lib

    assert b"sm_100a" in lib().frg_version()


MESHES = {
    "2d_periodic_p4": (lambda M: M.box2d(6, 5, perturb=0.1, seed=3), dict(order=4)),
    "2d_periodic_p1": (lambda M: M.box2d(3, 4, perturb=0.2, seed=9), dict(order=1)),
    "2d_bump_p3": (lambda M: M.bump2d(8, 4), dict(order=3)),
    "2d_bump_p5": (lambda M: M.bump2d(5, 3), dict(order=5)),
    "3d_periodic_p3": (lambda M: M.box3d(3, 4, 3, perturb=0.1, seed=4), dict(order=3)),
    "3d_char_p2": (lambda M: M.box3d(3, 3, 2, bcs={s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")},
                                     perturb=0.15, seed=5), dict(order=2)),
    "3d_mixed_p4": (lambda M: M.box3d(4, 3, 3, bcs={"zmin": "slip_wall", "zmax": "slip_wall"}, perturb=0.1, seed=6),
                    dict(order=4)),
}


@pytest.mark.parametrize("name", list(MESHES))
def test_geometry_matches_oracle(oracle, name):
    from fr_learn_b200 import mesh as M
    from fr_learn_b200.solver import inspect_geometry

    mk, kw = MESHES[name]
    m = mk(M)
    o = oracle.Oracle(oracle.params(nDims=m.nDims, **kw), m)
    for item in ("pos_spts", "JGinv_spts", "detJac_spts", "norm_fpts", "dA_fpts"):
        assert relerr(inspect_geometry(m, item, **kw), o.get(item)) < 1e-15, item
    fa = inspect_geometry(m, "faces", **kw)
    fb = o.faces()
    assert sorted(map(tuple, fa.tolist())) == sorted(map(tuple, fb.tolist()))


def test_geometry_matches_reference_golden(oracle):
    """The product's set-up on the golden meshes equals the reference's own
    metrics and face table."""
    from fr_learn_b200.mesh import Mesh
    from fr_learn_b200.solver import inspect_geometry

    g = np.load(os.path.join(ROOT, "tests", "golden", "reference_golden.npz"))
    for name in ("euler_p3_char_cfl", "ns_p3_walls"):
        pre = f"case/{name}/"
        m = Mesh(3, g[pre + "xv"], g[pre + "c2v"], g[pre + "bc"])
        P = int(g[pre + "setup"][0])
        assert relerr(inspect_geometry(m, "pos_spts", order=P), g[pre + "pos_spts"]) < 1e-15
        assert relerr(inspect_geometry(m, "detJac_spts", order=P), g[pre + "detJac_spts"]) < 1e-15
        assert relerr(inspect_geometry(m, "dA_fpts", order=P), g[pre + "dA_fpts"]) < 1e-15
        fa = inspect_geometry(m, "faces", order=P)
        assert sorted(map(tuple, fa.tolist())) == sorted(map(tuple, g[pre + "faces"].tolist()))


def test_periodic_mesh_needs_three_elements():
    from fr_learn_b200 import box2d, box3d

    with pytest.raises(ValueError):
        box2d(2, 5)
    with pytest.raises(ValueError):
        box3d(3, 2, 3)
    with pytest.raises(ValueError):
        box2d(4, 4, bcs={"xmin": "char"})  # periodic on one side only


def test_setup_rejects_bad_meshes():
    from fr_learn_b200 import FrgError, box2d
    from fr_learn_b200.solver import inspect_geometry

    m = box2d(4, 4, bcs={"xmin": "char", "xmax": "char", "ymin": "char", "ymax": "char"})
    m.bc[0, 3] = -1  # an outer face with no neighbour and no BC
    with pytest.raises(FrgError, match="no neighbour"):
        inspect_geometry(m, "faces", order=2)
    m2 = box2d(4, 4)
    m2.xv[0] = m2.xv[0][[1, 0, 3, 2]]  # mirrored element: negative Jacobian
    with pytest.raises(FrgError, match="Negative Jacobian"):
        inspect_geometry(m2, "detJac_spts", order=2)


def test_bump_mesh_shape():
    from fr_learn_b200 import bump2d

    m = bump2d(96, 32)
    assert m.xv.shape == (96 * 32, 9, 2)
    y = m.xv[:, :, 1]
    x = m.xv[:, :, 0]
    assert np.all(y >= 0.0625 * np.exp(-25 * x ** 2) - 1e-12)
    assert np.isclose(y.max(), 0.8)
    assert (m.bc[:, 0] == 8).sum() == 96 and (m.bc[:, 3] == 1).sum() == 32
