"""Ensemble mode on the GPU: independent cases advanced together in one
handle give, case by case, the same results as each case run alone (each
keeps its own CFL dt and time)."""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu


def _cases():
    from fr_learn_b200 import box2d

    return [box2d(3, 3, -10, 10, -10, 10, perturb=0.1, seed=1), box2d(5, 4, -10, 10, -10, 10, perturb=0.1, seed=2),
            box2d(4, 6, -8, 8, -10, 10, perturb=0.1, seed=3)]


def _vortex(pos, eps, uinf, gamma=1.4):
    """Isentropic vortex of strength eps in a freestream (uinf, rho = p = 1)."""
    x, y = pos[..., 0], pos[..., 1]
    f = 1.0 - (x * x + y * y)
    rho = (1.0 - eps * eps * (gamma - 1.0) / (8.0 * gamma * np.pi ** 2) * np.exp(f)) ** (1.0 / (gamma - 1.0))
    u = uinf[0] - eps * y / (2 * np.pi) * np.exp(f / 2)
    v = uinf[1] + eps * x / (2 * np.pi) * np.exp(f / 2)
    p = rho ** gamma
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)], axis=-1)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("dtType", [1, 0])
def test_ensemble_matches_cases_run_alone(precision, dtType):
    from fr_learn_b200 import Solver, concat_meshes

    cases = _cases()
    union, grp = concat_meshes(cases)
    kw = dict(order=3, riemannType=1, dtType=dtType, CFL=0.5, precision=precision)
    eps = [1.0, 3.0, 5.0]
    uinf = [(0.3, 0.2), (1.0, 1.0), (-0.5, 0.4)]
    fixed = np.array([1e-3, 2e-3, 1.5e-3])
    alone = []
    for k, m in enumerate(cases):
        s = Solver(m, **dict(kw, dt=fixed[k]))
        s.set("U_spts", _vortex(s.get("pos_spts"), eps[k], uinf[k]))
        s.update(6)
        alone.append((s.get("U_spts"), s.time, s.dt))
    e = Solver(union, **dict(kw, dt=fixed[0]))
    e.set_groups(grp, len(cases), fixed if dtType == 0 else None)
    pos = e.get("pos_spts")
    U0 = np.concatenate([_vortex(pos[:, grp == k], eps[k], uinf[k]) for k in range(len(cases))], axis=1)
    e.set("U_spts", U0)
    e.update(6)
    U = e.get("U_spts")
    t, dt = e.group_times()
    for k, (Ua, ta, dta) in enumerate(alone):
        Uk = U[:, grp == k]
        if precision == 0:
            # same kernels, same per-element arithmetic, same dt: identical
            assert np.array_equal(Uk, Ua), (k, relerr(Uk, Ua))
            assert t[k] == ta and dt[k] == dta
        else:
            assert relerr(Uk, Ua) < 1e-12
            assert t[k] == pytest.approx(ta, rel=1e-15) and dt[k] == pytest.approx(dta, rel=1e-15)


def test_ensemble_adjoint_matches_cases_alone():
    """FP64 adjoint of the entropy error in ensemble mode (fixed per-case dt):
    the gradient restricted to each case equals that case's own adjoint."""
    from fr_learn_b200 import Solver, concat_meshes

    cases = _cases()
    union, grp = concat_meshes(cases)
    kw = dict(order=2, riemannType=1, dtType=0)
    fixed = np.array([1e-3, 2e-3, 1.5e-3])
    lam = []
    for k, m in enumerate(cases):
        s = Solver(m, **dict(kw, dt=fixed[k]))
        s.set("U_spts", _vortex(s.get("pos_spts"), 2.0 + k, (0.5, 0.5)))
        s.adjoint_forward(5, 2)
        s.objective("entropy")
        lam.append(s.adjoint_backward()[0])
    e = Solver(union, **dict(kw, dt=fixed[0]))
    e.set_groups(grp, len(cases), fixed)
    pos = e.get("pos_spts")
    e.set("U_spts", np.concatenate([_vortex(pos[:, grp == k], 2.0 + k, (0.5, 0.5)) for k in range(3)], axis=1))
    e.adjoint_forward(5, 2)
    e.objective("entropy")
    lam_e = e.adjoint_backward()[0]
    for k in range(3):
        assert relerr(lam_e[:, grp == k], lam[k]) < 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_cross_order_ensemble_graph_matches_separate_updates(precision):
    """Two order groups (P=2, P=4), each the union of two cases, stepped by one
    graph launch per step give what each group's own frg_update gives."""
    from fr_learn_b200 import Ensemble, Solver, concat_meshes

    cases = _cases()
    outs = []
    for use_ens in (False, True):
        solvers = []
        for P, idx in ((2, (0, 1)), (4, (1, 2))):
            union, grp = concat_meshes([cases[i] for i in idx])
            s = Solver(union, order=P, riemannType=1, dtType=1, CFL=0.5, precision=precision)
            s.set_groups(grp, 2)
            pos = s.get("pos_spts")
            s.set("U_spts", np.concatenate([_vortex(pos[:, grp == k], 2.0 + k, (0.5, -0.3)) for k in range(2)],
                                           axis=1))
            solvers.append(s)
        if use_ens:
            ens = Ensemble(solvers)
            ens.update(3)
            ens.update(4)
            ens.close()
        else:
            for s in solvers:
                s.update(7)
        outs.append([(s.get("U_spts"), s.group_times()) for s in solvers])
    for (Ua, (ta, da)), (Ub, (tb, db)) in zip(outs[0], outs[1]):
        assert np.array_equal(Ua, Ub)
        assert np.array_equal(ta, tb) and np.array_equal(da, db)


@pytest.mark.parametrize("precision", [0, 1])
def test_ensemble_persistent_variants_multi_tile(precision):
    """Ensemble mode with the persistent stage kernels on cases large enough
    that a block walks two or three tiles, with tiles that straddle two cases
    (each element's group takes its own dt minimum in the deferred per-tile
    dt): every tile variant gives, case by case, the results of the case run
    alone."""
    from fr_learn_b200 import Solver, box2d, concat_meshes

    cases = [box2d(60, 57, -10, 10, -10, 10, perturb=0.1, seed=51), box2d(53, 65, -10, 10, -10, 10, perturb=0.1, seed=52),
             box2d(58, 61, -8, 8, -10, 10, perturb=0.1, seed=53)]
    union, grp = concat_meshes(cases)
    kw = dict(order=3, riemannType=1, dtType=1, CFL=0.5, precision=precision)
    eps = [1.0, 3.0, 5.0]
    uinf = [(0.3, 0.2), (1.0, 1.0), (-0.5, 0.4)]
    nsteps = 4
    alone = []
    for k, m in enumerate(cases):
        s = Solver(m, **kw)
        s.set("U_spts", _vortex(s.get("pos_spts"), eps[k], uinf[k]))
        s.update(nsteps)
        alone.append((s.get("U_spts"), s.time, s.dt))
        s.close()
    nvar = Solver(union, **kw).tile_variant_count()
    for v in range(nvar):
        e = Solver(union, **kw)
        e.set_tile_variant(v)
        e.set_groups(grp, len(cases), None)
        pos = e.get("pos_spts")
        e.set("U_spts", np.concatenate([_vortex(pos[:, grp == k], eps[k], uinf[k]) for k in range(len(cases))],
                                       axis=1))
        e.update(nsteps)
        U = e.get("U_spts")
        t, dt = e.group_times()
        for k, (Ua, ta, dta) in enumerate(alone):
            Uk = U[:, grp == k]
            if precision == 0:
                assert np.array_equal(Uk, Ua), (v, k, relerr(Uk, Ua))
                assert t[k] == ta and dt[k] == dta, (v, k)
            else:
                assert relerr(Uk, Ua) < 1e-12, (v, k)
                assert t[k] == pytest.approx(ta, rel=1e-15) and dt[k] == pytest.approx(dta, rel=1e-15), (v, k)
        e.close()
