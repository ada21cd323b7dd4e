"""The allocation-free residual entry point (frg_calc_residual_noalloc).

It serves callers that cannot allocate device memory at the time they need a
residual (all device memory owned by another manager, or planned up front).
The test calls it through the C ABI with caller-owned device buffers and
checks, on two calls in a row with different states, that it returns the
same divF as the regular solver::calcResidual path (frg_calc_residual), to
the FP64 parity tolerance of the other tests.  This file sorts last so that a
run stopping at the first failure has already run every other test.
"""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _to_dev_layout(a):
    # reference layout [pt][ele][field] -> device layout [field][pt][ele]
    return np.ascontiguousarray(np.transpose(a, (2, 0, 1)))


def _case(name):
    import numpy as np

    from fr_learn_b200 import box2d, box3d

    if name == "euler2d":
        return box2d(10, 9, -10, 10, -10, 10, perturb=0.1, seed=11), 1, 0.0, dict(order=4, riemannType=1,
                                                                                   dtType=1, CFL=0.5)
    if name == "ns2d":
        return box2d(7, 6, -10, 10, -10, 10, perturb=0.1, seed=12), 1, 0.0, dict(
            order=3, riemannType=1, viscous=1, mu_inf=0.01, prandtl=0.72, fixVis=1, penFact=0.5, tau=1.0,
            dtType=1, CFL=0.3)
    # 3D Navier-Stokes with an LDG penalty: the second projected-flux array
    return box3d(3, 4, 3, (0, 0, 0), (2 * np.pi,) * 3, perturb=0.05, seed=14), 10, 0.1, dict(
        order=3, viscous=1, mu_inf=1.0 / 1600, prandtl=0.71, fixVis=1, penFact=0.3, tau=1.0, dtType=0, dt=1e-3)


@pytest.mark.parametrize("name", ["euler2d", "ns2d", "ns3d_penalty"])
@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_residual_matches_calc_residual(precision, name):
    import torch

    from fr_learn_b200 import Solver

    mesh, ic, a0, kw = _case(name)
    s = Solver(mesh, precision=precision, **kw)
    s.setInitialCondition(ic, a0)
    dev = torch.device("cuda", torch.cuda.current_device())
    nV, nS, nE = s.nFields, s.nSpts, s.nEles
    divF_dev = torch.full((nV, nS, nE), float("nan"), dtype=torch.float64, device=dev)
    for call in range(2):
        if call == 1:
            s.update(3)  # a different state for the second call
        U = s.get("U_spts")
        s.calcResidual(0)
        ref = s.get("divF_spts", 0)
        U_dev = torch.from_numpy(_to_dev_layout(U)).to(dev)
        s.sync()
        s.calcResidual_noalloc(U_dev.data_ptr(), divF_dev.data_ptr())
        s.sync()
        got = np.transpose(divF_dev.cpu().numpy(), (1, 2, 0))
        assert np.isfinite(got).all()
        assert relerr(got, ref) < FP64_TOL


def test_noalloc_rejects_oversized_mesh():
    import torch

    from fr_learn_b200 import FrgError, Solver, box2d

    # 4 * 24 * 200*120 traces * 8 B = 18.4 MB > 16 MiB scratch
    mesh = box2d(200, 120, -10, 10, -10, 10)
    s = Solver(mesh, order=5, riemannType=1)
    dev = torch.device("cuda", torch.cuda.current_device())
    U = torch.zeros((s.nFields, s.nSpts, s.nEles), dtype=torch.float64, device=dev)
    out = torch.zeros_like(U)
    with pytest.raises(FrgError, match="scratch"):
        s.calcResidual_noalloc(U.data_ptr(), out.data_ptr())


def test_noalloc_viscous_buffers_count_toward_the_limit():
    """3D Navier-Stokes, 14^3 hexes at P = 2: the traces alone (5.9 MB) fit,
    and without an LDG penalty traces plus one projected-flux array fit too;
    with a penalty the second projected-flux array pushes the total past
    16 MiB and the call is rejected."""
    import numpy as np
    import torch

    from fr_learn_b200 import FrgError, Solver, box3d

    mesh = box3d(14, 14, 14, (0, 0, 0), (2 * np.pi,) * 3)
    kw = dict(order=2, viscous=1, mu_inf=1.0 / 1600, prandtl=0.71, fixVis=1, tau=1.0, dtType=0, dt=1e-3)
    dev = torch.device("cuda", torch.cuda.current_device())
    ok = Solver(mesh, penFact=0.0, **kw)
    ok.setInitialCondition(10, 0.1)
    U = torch.from_numpy(_to_dev_layout(ok.get("U_spts"))).to(dev)
    out = torch.zeros_like(U)
    ok.sync()
    ok.calcResidual_noalloc(U.data_ptr(), out.data_ptr())
    ok.sync()
    ok.calcResidual(0)
    assert relerr(np.transpose(out.cpu().numpy(), (1, 2, 0)), ok.get("divF_spts", 0)) < FP64_TOL
    pen = Solver(mesh, penFact=0.3, **kw)
    with pytest.raises(FrgError, match="scratch"):
        pen.calcResidual_noalloc(U.data_ptr(), out.data_ptr())
