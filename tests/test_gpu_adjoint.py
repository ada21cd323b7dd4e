"""Discrete adjoint on the GPU against finite differences.

* residual VJP: <gbar, dR/dU delta> by central differences of calcResidual,
  and the boundary-state parameter column, for periodic / wall+char / 3D /
  advection configurations;
* the reverse RK sweep with checkpoints: dJ/dU_0 and dJ/dMach of the wall
  pressure integral over the bump against central differences of the
  forward solver (step 1e-6, agreement to 1e-5);
* the same gradient against finite differences assembled from the CPU oracle
  (the reference's algorithm restated), for the entropy-error objective.
"""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

GAMMA = 1.4


def _cases():
    from fr_learn_b200 import box2d, box3d, bump2d

    char6 = {s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    c = np.sqrt(GAMMA)
    return {
        "vortex2d_p3_roe": (box2d(4, 4, -5, 5, -5, 5, perturb=0.1, seed=3), 1,
                            dict(order=3, riemannType=1)),
        "bump2d_p2_roe_char_slip": (bump2d(6, 3), 0,
                                    dict(order=2, riemannType=1, uBound=0.5 * c, pBound=1.0)),
        "bump2d_p3_rusanov": (bump2d(5, 3), 0, dict(order=3, riemannType=0, uBound=0.4 * c, pBound=1.0)),
        "euler3d_p2_char": (box3d(3, 3, 3, (-2, -2, -2), (2, 2, 2), bcs=char6, perturb=0.1, seed=1), 1,
                            dict(order=2, uBound=0.3, pBound=1.0 / GAMMA)),
        "advection2d_p3": (box2d(4, 3, -5, 5, -5, 5, perturb=0.1, seed=5), 0, dict(order=3, equation=0)),
    }


def _solver(mesh, ic, **kw):
    from fr_learn_b200 import Solver

    s = Solver(mesh, dtType=0, dt=1e-3, **kw)
    s.setInitialCondition(ic)
    return s


def _perturbed_state(s, rng, amp=1e-2):
    U = s.get("U_spts")
    scale = np.abs(U).max(axis=(0, 1), keepdims=True)
    return U * (1.0 + amp * rng.standard_normal(U.shape)) + 0.1 * amp * scale * rng.standard_normal(U.shape)


def _residual(s, U):
    s.set("U_spts", U)
    s.calcResidual(0)
    return s.get("divF_spts", 0)


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_residual_vjp_matches_central_differences(name):
    mesh, ic, kw = _cases()[name]
    rng = np.random.default_rng(7)
    s = _solver(mesh, ic, **kw)
    U = _perturbed_state(s, rng)
    gbar = rng.standard_normal(U.shape)
    delta = rng.standard_normal(U.shape) * np.abs(U).max(axis=(0, 1), keepdims=True)
    s.set("U_spts", U)
    theta = None
    if kw.get("uBound") is not None and "bump" in name:
        theta = np.array([0.0, np.sqrt(GAMMA), 0.0, 0.0, 0.0])  # d(u_B)/dMach
    ubar, tbar = s.residual_vjp(gbar, theta)
    eps = 1e-6
    fd = np.sum(gbar * (_residual(s, U + eps * delta) - _residual(s, U - eps * delta))) / (2 * eps)
    adj = np.sum(ubar * delta)
    bound = np.linalg.norm(ubar) * np.linalg.norm(delta)  # |<ubar, delta>| <= bound
    assert abs(fd - adj) <= 1e-7 * abs(adj) + 1e-10 * bound, (fd, adj, bound)
    if theta is not None:
        # central differences over the boundary Mach number at a fixed state
        M = kw["uBound"] / np.sqrt(GAMMA)
        R = []
        for sg in (1, -1):
            k2 = dict(kw, uBound=(M + sg * eps) * np.sqrt(GAMMA))
            s2 = _solver(mesh, ic, **k2)
            R.append(_residual(s2, U))
        fdt = np.sum(gbar * (R[0] - R[1])) / (2 * eps)
        assert abs(fdt - tbar) <= 1e-6 * max(abs(tbar), 1e-8), (fdt, tbar)


def _wallp_after(mesh, kw, U0, nsteps):
    s = _solver(mesh, 0, **kw)
    s.set("U_spts", U0)
    s.update(nsteps)
    return s.objective("wall_pressure")[0]


def _freestream_dU_dM(U0, c):
    """d(freestream state)/dMach for rho, p fixed, velocity (M c, 0)."""
    rho = U0[..., 0]
    u = U0[..., 1] / rho
    d = np.zeros_like(U0)
    d[..., 1] = rho * c
    d[..., 3] = rho * u * c
    return d


@pytest.mark.parametrize("timeType,nsteps,every", [(4, 7, 3), (2, 5, 5), (0, 4, 2), (4, 6, 0)])
def test_adjoint_rk_matches_central_differences(timeType, nsteps, every):
    """Bump channel (P=2, Roe, char inlet/outlet, slip lower wall, symmetry
    top), J = wall pressure integral after nsteps; gradients with respect to
    the initial state (a random direction) and to the freestream Mach number.
    every = 0: the forward run keeps all stage states (no recomputation)."""
    from fr_learn_b200 import bump2d

    c = np.sqrt(GAMMA)
    M = 0.5
    mesh = bump2d(8, 3, bc_top="symmetry")
    kw = dict(order=2, riemannType=1, uBound=M * c, pBound=1.0, timeType=timeType)
    s = _solver(mesh, 0, **kw)
    U0 = s.get("U_spts")
    s.adjoint_forward(nsteps, every)
    J, _ = s.objective("wall_pressure")
    theta = np.array([0.0, c, 0.0, 0.0, 0.0])
    lam0, tbar = s.adjoint_backward(None, theta)
    assert J == pytest.approx(_wallp_after(mesh, kw, U0, nsteps), rel=1e-13)
    # the solution is left at U_N
    s2 = _solver(mesh, 0, **kw)
    s2.update(nsteps)
    assert relerr(s.get("U_spts"), s2.get("U_spts")) < 1e-13
    assert s.time == pytest.approx(s2.time, rel=1e-14)

    rng = np.random.default_rng(11)
    delta = rng.standard_normal(U0.shape) * np.abs(U0).max(axis=(0, 1), keepdims=True)
    eps = 1e-6
    fd = (_wallp_after(mesh, kw, U0 + eps * delta, nsteps) - _wallp_after(mesh, kw, U0 - eps * delta, nsteps)) / (
        2 * eps)
    adj = float(np.sum(lam0 * delta))
    assert abs(fd - adj) <= 1e-5 * abs(adj), (fd, adj)

    # Mach: boundary state and the freestream initial state move together
    Jm = []
    for sg in (1, -1):
        k2 = dict(kw, uBound=(M + sg * eps) * c)
        s3 = _solver(mesh, 0, **k2)
        s3.update(nsteps)
        Jm.append(s3.objective("wall_pressure")[0])
    fdM = (Jm[0] - Jm[1]) / (2 * eps)
    adjM = float(np.sum(lam0 * _freestream_dU_dM(U0, c))) + tbar
    assert abs(fdM - adjM) <= 1e-5 * abs(adjM), (fdM, adjM)


def _entropy_numpy(U, detJ, P):
    """The entropy-error integral of a state in reference layout."""
    x, w = np.polynomial.legendre.leggauss(P + 1)
    ws = np.outer(w, w).ravel()  # s = i + (P+1) j
    rho = U[..., 0]
    ke = (U[..., 1] ** 2 + U[..., 2] ** 2) / rho
    p = (GAMMA - 1) * (U[..., 3] - 0.5 * ke)
    err = p / rho ** GAMMA - 1.0
    return float(np.sum(ws[:, None] * detJ * err))


def test_adjoint_matches_oracle_finite_differences(oracle):
    """Periodic vortex (strength 2), P=3, Roe, RK4, 6 steps; J = entropy error.
    dJ/dU_0 along two random directions from the GPU adjoint against central
    differences of the CPU oracle's forward run."""
    from fr_learn_b200 import box2d

    mesh = box2d(4, 4, -5, 5, -5, 5, perturb=0.1, seed=9)
    kw = dict(order=3, riemannType=1, rhoBound=1.0, pBound=1.0)
    nsteps = 6
    s = _solver(mesh, 11, **kw)
    s.setInitialCondition(11, 2.0)
    U0 = s.get("U_spts")
    detJ = s.get("detJac_spts")
    s.adjoint_forward(nsteps, 4)
    J, _ = s.objective("entropy")
    lam0, _ = s.adjoint_backward()

    p = oracle.params(nDims=2, dtType=0, dt=1e-3, **kw)

    def J_oracle(U):
        o = oracle.Oracle(p, mesh)
        o.set("U_spts", U)
        o.update(nsteps)
        return _entropy_numpy(o.U(), detJ, 3)

    assert J == pytest.approx(J_oracle(U0), rel=1e-8, abs=1e-12)
    rng = np.random.default_rng(5)
    eps = 1e-6
    for _ in range(2):
        delta = rng.standard_normal(U0.shape) * np.abs(U0).max(axis=(0, 1), keepdims=True)
        fd = (J_oracle(U0 + eps * delta) - J_oracle(U0 - eps * delta)) / (2 * eps)
        adj = float(np.sum(lam0 * delta))
        assert abs(fd - adj) <= 1e-5 * abs(adj), (fd, adj)


def test_autograd_binding_matches_central_differences():
    """A torch loss of the final state, differentiated through FRSteps (the
    adjoint as a torch.autograd.Function), against central differences."""
    import torch

    from fr_autograd import FRSteps
    from fr_learn_b200 import box2d

    mesh = box2d(4, 3, -5, 5, -5, 5, perturb=0.1, seed=4)
    kw = dict(order=3, riemannType=0)
    s = _solver(mesh, 1, **kw)
    U0 = torch.from_numpy(s.get("U_spts")).requires_grad_(True)
    W = torch.from_numpy(np.random.default_rng(2).standard_normal(tuple(U0.shape)))

    def loss(U):
        return (W * U * U).sum()

    L = loss(FRSteps.apply(U0, s, 5, 2))
    L.backward()
    g = U0.grad.numpy()
    delta = np.random.default_rng(3).standard_normal(g.shape)
    eps = 1e-6
    Lp = []
    for sg in (1, -1):
        s2 = _solver(mesh, 1, **kw)
        s2.set("U_spts", U0.detach().numpy() + sg * eps * delta)
        s2.update(5)
        Lp.append(float(loss(torch.from_numpy(s2.get("U_spts")))))
    fd = (Lp[0] - Lp[1]) / (2 * eps)
    adj = float(np.sum(g * delta))
    assert abs(fd - adj) <= 1e-6 * abs(adj), (fd, adj)


def test_checkpointed_and_stored_sweeps_agree():
    """Checkpoint intervals 1, 3, 'keep everything' and the automatic choice
    give the same dJ/dU_0."""
    from fr_learn_b200 import bump2d

    c = np.sqrt(GAMMA)
    mesh = bump2d(6, 3, bc_top="symmetry")
    kw = dict(order=3, riemannType=1, uBound=0.5 * c, pBound=1.0)
    out = []
    for every in (1, 3, 0, -1):
        s = _solver(mesh, 0, **kw)
        s.adjoint_forward(8, every)
        # the automatic strategy keeps every stage state of a run this small
        assert s.adjoint_mode() == (0 if every <= 0 else every)
        s.objective("wall_pressure")
        out.append(s.adjoint_backward(None, np.array([0.0, c, 0, 0, 0]))[0])
        # a second sweep replays the captured segment graphs (both slot sets of
        # the overlapped recompute / reverse) and must give the same bits
        assert np.array_equal(s.adjoint_backward(None, np.array([0.0, c, 0, 0, 0]))[0], out[-1])
    assert relerr(out[1], out[0]) < 1e-12 and relerr(out[2], out[0]) < 1e-12
    assert np.array_equal(out[3], out[2])


# ---- viscous (LDG) residuals: the three-pass viscous adjoint
def _visc_cases():
    from fr_learn_b200 import box2d, box3d, bump2d

    c = np.sqrt(GAMMA)
    ns = dict(viscous=1, mu_inf=0.05, prandtl=0.72, fixVis=1, tau=1.0)
    return {
        "ns2d_p3_roe_periodic": (box2d(4, 4, -5, 5, -5, 5, perturb=0.1, seed=13), 1,
                                 dict(order=3, riemannType=1, penFact=0.5, **ns)),
        "ns2d_p2_walls_char": (bump2d(5, 3, bc_wall="adiabatic_noslip", bc_top="isothermal_noslip"), 0,
                               dict(order=2, riemannType=0, penFact=0.3, TWall=1.0, RGas=1.0 / GAMMA,
                                    uBound=0.3 * c, pBound=1.0, **ns)),
        "ns2d_p2_sutherland_slip": (bump2d(5, 3), 0,
                                    dict(order=2, riemannType=1, penFact=0.0, uBound=0.4 * c, pBound=1.0,
                                         viscous=1, mu_inf=0.05, prandtl=0.71, fixVis=0, c_sth=0.41, rt_inf=2.5,
                                         tau=1.0)),
        "ns3d_p2_periodic": (box3d(3, 3, 3, (0, 0, 0), (2 * np.pi,) * 3, perturb=0.05, seed=14), 10,
                             dict(order=2, penFact=0.0, **ns)),
        "ns3d_p2_penalty_walls": (box3d(3, 3, 3, (-2, -2, -1), (2, 2, 1),
                                        bcs={"zmin": "adiabatic_noslip", "zmax": "isothermal_noslip"},
                                        perturb=0.1, seed=15), 1,
                                  dict(order=2, penFact=0.3, TWall=1.0, RGas=1.0 / GAMMA, **ns)),
        "advdiff2d_p3": (box2d(4, 4, perturb=0.1, seed=16), 0,
                         dict(order=3, equation=0, viscous=1, diffD=0.05, penFact=0.2, tau=1.0)),
    }


@pytest.mark.parametrize("name", list(_visc_cases().keys()))
def test_viscous_residual_vjp_matches_central_differences(name):
    mesh, ic, kw = _visc_cases()[name]
    rng = np.random.default_rng(11)
    s = _solver(mesh, ic, **kw) if ic != 10 else None
    if s is None:
        from fr_learn_b200 import Solver

        s = Solver(mesh, dtType=0, dt=1e-3, **kw)
        s.setInitialCondition(10, 0.2)
    U = _perturbed_state(s, rng)
    gbar = rng.standard_normal(U.shape)
    delta = rng.standard_normal(U.shape) * np.abs(U).max(axis=(0, 1), keepdims=True)
    s.set("U_spts", U)
    theta = None
    if "char" in name or "slip" in name:
        theta = np.array([0.0, np.sqrt(GAMMA), 0.0, 0.0, 0.0])  # d(u_B)/dMach
    ubar, tbar = s.residual_vjp(gbar, theta)
    eps = 1e-6
    fd = np.sum(gbar * (_residual(s, U + eps * delta) - _residual(s, U - eps * delta))) / (2 * eps)
    adj = np.sum(ubar * delta)
    bound = np.linalg.norm(ubar) * np.linalg.norm(delta)
    assert abs(fd - adj) <= 1e-6 * abs(adj) + 1e-10 * bound, (fd, adj, bound)
    if theta is not None:
        M = kw["uBound"] / np.sqrt(GAMMA)
        R = []
        for sg in (1, -1):
            k2 = dict(kw, uBound=(M + sg * eps) * np.sqrt(GAMMA))
            s2 = _solver(mesh, ic, **k2)
            R.append(_residual(s2, U))
        fdt = np.sum(gbar * (R[0] - R[1])) / (2 * eps)
        assert abs(fdt - tbar) <= 1e-5 * max(abs(tbar), 1e-8), (fdt, tbar)


@pytest.mark.parametrize("every", [3, 0])
def test_viscous_adjoint_rk_matches_central_differences(every):
    """Navier-Stokes channel over the bump (P = 2, Rusanov, LDG with a
    penalty, adiabatic lower wall, isothermal top, characteristic in / out),
    J = entropy-error integral after 6 RK4 steps: dJ/dU_0 along a random
    direction and dJ/dMach against central differences of the forward solver."""
    from fr_learn_b200 import bump2d

    c = np.sqrt(GAMMA)
    M = 0.3
    mesh = bump2d(6, 3, bc_wall="adiabatic_noslip", bc_top="isothermal_noslip")
    kw = dict(order=2, riemannType=0, viscous=1, mu_inf=0.05, prandtl=0.72, fixVis=1, tau=1.0, penFact=0.3,
              TWall=1.0, RGas=1.0 / GAMMA, uBound=M * c, pBound=1.0, timeType=4)
    nsteps = 6
    rng = np.random.default_rng(5)
    s = _solver(mesh, 0, **kw)
    U0 = _perturbed_state(s, rng, amp=2e-3)
    s.set("U_spts", U0)
    s.adjoint_forward(nsteps, every)
    J, _ = s.objective("entropy")
    theta = np.array([0.0, c, 0.0, 0.0, 0.0])
    lam0, tbar = s.adjoint_backward(None, theta)

    def J_of(U, Mach):
        s2 = _solver(mesh, 0, **dict(kw, uBound=Mach * c))
        s2.set("U_spts", U)
        s2.update(nsteps)
        return s2.objective("entropy")[0]

    eps = 1e-6
    d = rng.standard_normal(U0.shape) * np.abs(U0).max(axis=(0, 1), keepdims=True)
    fd = (J_of(U0 + eps * d, M) - J_of(U0 - eps * d, M)) / (2 * eps)
    adj = float(np.sum(lam0 * d))
    assert abs(fd - adj) <= 1e-5 * abs(adj), (fd, adj)
    fdm = (J_of(U0, M + eps) - J_of(U0, M - eps)) / (2 * eps)
    assert abs(fdm - tbar) <= 1e-5 * abs(fdm), (fdm, tbar)
