"""Failure detection of the device path, made on the host.

The reference stops with fatalError when the residual monitor finds a NaN
(src/output.cpp:833-841) or when dt falls below 1e-13 (:823-824).  Here the
kernels set a flag word and frg_update returns FRG_ERR_NAN / FRG_ERR_DT.
The failures are planted in the inputs (a NaN in the uploaded state, a CFL
number or fixed dt so small that dt underflows the threshold); no GPU fault
is involved.  After the error the handle stays usable: a valid state
uploaded again steps normally.
"""
import numpy as np
import pytest

from fr_learn_b200 import FRG_FP64, FRG_MIXED, FrgError, Solver, box2d, box3d

pytestmark = pytest.mark.gpu

ERR_NAN, ERR_DT = 3, 5


def _cases():
    return {
        "euler2d_tma": (box2d(9, 7, -10, 10, -10, 10, perturb=0.1, seed=31), 1,
                        dict(order=4, riemannType=1)),
        "euler3d": (box3d(3, 3, 3, perturb=0.1, seed=32), 10, dict(order=2)),
        "ns3d_visc": (box3d(3, 3, 3, (0, 0, 0), (2 * np.pi,) * 3, perturb=0.05, seed=33), 10,
                      dict(order=3, viscous=1, mu_inf=1.0 / 1600, prandtl=0.71, fixVis=1)),
    }


@pytest.mark.parametrize("precision", [FRG_FP64, FRG_MIXED])
@pytest.mark.parametrize("name", list(_cases()))
def test_nan_in_state_reports_err_nan(name, precision):
    mesh, ic, kw = _cases()[name]
    a0 = 0.1 if ic == 10 else 0.0
    s = Solver(mesh, precision=precision, dtType=0, dt=1e-3, **kw)
    s.setInitialCondition(ic, a0)
    good = s.get("U_spts")
    bad = good.copy()
    bad[3, mesh.nEles // 2, 0] = np.nan
    s.set("U_spts", bad)
    with pytest.raises(FrgError) as ei:
        s.update(1)
    assert ei.value.code == ERR_NAN
    # the flag is cleared and the handle still works
    s.set("U_spts", good)
    s.update(2)
    assert np.isfinite(s.get("U_spts")).all()


@pytest.mark.parametrize("name", list(_cases()))
def test_cfl_dt_underflow_reports_err_dt(name):
    mesh, ic, kw = _cases()[name]
    a0 = 0.1 if ic == 10 else 0.0
    s = Solver(mesh, dtType=1, CFL=1e-16, **kw)
    s.setInitialCondition(ic, a0)
    with pytest.raises(FrgError) as ei:
        s.update(3)
    assert ei.value.code == ERR_DT


def test_fixed_dt_underflow_reports_err_dt():
    mesh, ic, kw = _cases()["euler2d_tma"]
    s = Solver(mesh, dtType=0, dt=1e-14, **kw)
    s.setInitialCondition(ic)
    with pytest.raises(FrgError) as ei:
        s.update(1)
    assert ei.value.code == ERR_DT


def test_nan_reported_through_host_update():
    """frg_update_host (upload, steps, download) reports the NaN too, and
    hands back the failed step's state as the reference's array holds it."""
    mesh, ic, kw = _cases()["euler2d_tma"]
    s = Solver(mesh, dtType=0, dt=1e-3, **kw)
    s.setInitialCondition(ic)
    U = s.get("U_spts")
    U[0, 0, 3] = np.nan
    Uh = np.ascontiguousarray(U)
    with pytest.raises(FrgError) as ei:
        s.update_host(Uh, 1)
    assert ei.value.code == ERR_NAN
    assert np.isnan(Uh).any() and np.array_equal(Uh, s.get("U_spts"), equal_nan=True)


@pytest.mark.parametrize("precision", [FRG_FP64, FRG_MIXED])
@pytest.mark.parametrize("name,extra", [("euler2d_tma", dict(dtType=1, CFL=0.5)), ("ns3d_visc", dict(dtType=1, CFL=0.3)),
                                        ("euler2d_tma", dict(dtType=1, CFL=0.5, timeType=0))])
def test_host_update_matches_device_update(name, extra, precision):
    """frg_update_host (one synchronisation per call) gives bit for bit what
    an upload, frg_update and a download give, over consecutive calls (the
    CFL dt carried between them); Forward Euler with CFL dt takes the
    unfused path."""
    mesh, ic, kw = _cases()[name]
    a0 = 0.1 if ic == 10 else 0.0
    a = Solver(mesh, precision=precision, **kw, **extra)
    b = Solver(mesh, precision=precision, **kw, **extra)
    for s in (a, b):
        s.setInitialCondition(ic, a0)
    Uh = np.ascontiguousarray(a.get("U_spts"))
    for n in (1, 3, 2):
        a.update_host(Uh, n)
        b.set("U_spts", b.get("U_spts"))
        b.update(n)
        assert np.array_equal(Uh, b.get("U_spts")), n
        assert a.time == b.time and a.dt == b.dt
