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


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_residual_matches_calc_residual(precision):
    import torch

    from fr_learn_b200 import Solver, box2d

    mesh = box2d(10, 9, -10, 10, -10, 10, perturb=0.1, seed=11)
    s = Solver(mesh, order=4, riemannType=1, dtType=1, CFL=0.5, precision=precision)
    s.setInitialCondition(1)
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
