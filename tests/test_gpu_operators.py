"""frg_set_operators: the reference's own oper::setupOperators matrices
(tests/golden/reference_golden.npz, made from the FlurryPP sources) handed
to the device path.  Matrices of another correction scheme switch the
solver to that scheme (the residual then matches the oracle run with it);
matrices that are no scheme's FR operators are rejected."""
import os

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.npz")


def _ref_ops(g, d, P, v):
    pre = f"ops/{d}d_p{P}_v{v}/"
    E = g[pre + "spts_to_fpts"]
    C = g[pre + "correction"]
    D = np.stack([g[pre + f"grad_spts_{k}"] for k in range(d)])
    Efn = np.stack([g[pre + f"extrapolateFn_{k}"] for k in range(d)])
    return E, D, C, Efn


@pytest.mark.parametrize("d,v", [(2, 2), (2, 1), (3, 2), (2, 0)])
def test_reference_operators_select_the_scheme(oracle, d, v):
    from fr_learn_b200 import Solver, box2d, box3d

    g = np.load(GOLD)
    P = 3
    mesh = box2d(6, 5, -10, 10, -10, 10, perturb=0.1, seed=61) if d == 2 else box3d(3, 3, 3, perturb=0.1, seed=62)
    ic = 1 if d == 2 else 10
    a0 = 0.0 if d == 2 else 0.1
    s = Solver(mesh, order=P, riemannType=1 if d == 2 else 0, dtType=0, dt=1e-3)
    s.set_operators(P, *_ref_ops(g, d, P, v))
    s.setInitialCondition(ic, a0)
    s.update(2)
    s.calcResidual(0)
    o = oracle.Oracle(oracle.params(nDims=d, order=P, riemannType=1 if d == 2 else 0, dtType=0, dt=1e-3,
                                    vcjhScheme=v), mesh)
    o.set_ic(ic, a0)
    o.update(2)
    o.calc_residual(0)
    assert relerr(s.get("U_spts"), o.U()) < 1e-12
    assert relerr(s.get("divF_spts", 0), o.divF(0)) < 1e-12
    assert np.array_equal(s.operator(3), g[f"ops/{d}d_p{P}_v{v}/correction"])


def test_foreign_matrices_are_rejected():
    from fr_learn_b200 import FrgError, Solver, box2d

    g = np.load(GOLD)
    s = Solver(box2d(4, 4), order=3)
    E, D, C, Efn = _ref_ops(g, 2, 3, 0)
    with pytest.raises(FrgError, match="not the FR operators"):
        s.set_operators(3, E, D, 1.01 * C, Efn)
    with pytest.raises(FrgError, match="order"):
        s.set_operators(2, *_ref_ops(g, 2, 2, 0))
