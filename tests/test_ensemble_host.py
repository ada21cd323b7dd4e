"""Ensemble mode, host side: the union mesh of independent cases has exactly
the cases' own face pairings (offset per case) and geometry."""
import numpy as np

from fr_learn_b200 import box2d, concat_meshes
from fr_learn_b200.solver import inspect_geometry


def test_union_mesh_keeps_cases_apart():
    cases = [box2d(3, 3, -10, 10, -10, 10, perturb=0.1, seed=1), box2d(4, 3, -10, 10, -10, 10, perturb=0.1, seed=2),
             box2d(5, 5, -10, 10, -10, 10, perturb=0.1, seed=3)]
    union, grp = concat_meshes(cases)
    assert union.nEles == sum(m.nEles for m in cases)
    assert np.array_equal(grp, np.repeat(np.arange(3), [m.nEles for m in cases]))
    kw = dict(order=3)
    fu = inspect_geometry(union, "faces", **kw)
    off, rows = 0, []
    for m in cases:
        f = inspect_geometry(m, "faces", **kw).copy()
        for col in (0, 2):
            f[:, col] = np.where(f[:, col] >= 0, f[:, col] + off, f[:, col])
        rows.append(f)
        off += m.nEles
    ref = np.concatenate(rows)
    # same set of face rows (element, face, element, face, rotation, bc)
    key = lambda a: sorted(map(tuple, a.tolist()))
    assert key(fu) == key(ref)
    # no face joins two cases
    inter = fu[fu[:, 2] >= 0]
    assert np.all(grp[inter[:, 0]] == grp[inter[:, 2]])
    du = inspect_geometry(union, "detJac_spts", **kw).reshape(-1, union.nEles)
    parts = [inspect_geometry(m, "detJac_spts", **kw).reshape(-1, m.nEles) for m in cases]
    assert np.array_equal(du, np.concatenate(parts, axis=1))
