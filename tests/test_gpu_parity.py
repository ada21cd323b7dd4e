"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64 mode: the bar is 1e-12 relative (max-norm over the array, relative to
the array's max) for a residual and for multi-step updates.  Mixed mode: the
stated bound is checked in test_mixed_precision_bound.
"""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def pair(oracle, mesh, ic, a0=0.0, **kw):
    from fr_learn_b200 import Solver

    g = Solver(mesh, **kw)
    okw = {k: v for k, v in kw.items() if k != "precision"}
    o = oracle.Oracle(oracle.params(nDims=mesh.nDims, **okw), mesh)
    o.set_ic(ic, a0)
    g.setInitialCondition(ic, a0)
    assert relerr(g.get("U_spts"), o.U()) == 0.0
    return g, o


def cases():
    from fr_learn_b200 import box2d, box3d, bump2d

    char6 = {s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    return {
        "vortex2d_p4_roe": (box2d(8, 8, -10, 10, -10, 10, perturb=0.1, seed=7), 1,
                            dict(order=4, riemannType=1, dtType=1, CFL=0.5)),
        "vortex2d_p3_rusanov": (box2d(6, 7, -10, 10, -10, 10, perturb=0.1, seed=8), 1,
                                dict(order=3, riemannType=0, dtType=0, dt=2e-3)),
        "vortex2d_p5_roe": (box2d(5, 5, -10, 10, -10, 10, perturb=0.05, seed=9), 1,
                            dict(order=5, riemannType=1, dtType=1, CFL=0.3)),
        "advection2d_p3": (box2d(8, 8), 0, dict(order=3, equation=0, dt=1e-3)),
        "advection2d_p2_cfl": (box2d(6, 5, perturb=0.1, seed=1), 0, dict(order=2, equation=0, dtType=1, CFL=0.5)),
        "bump2d_p3_roe": (bump2d(12, 4), 0, dict(order=3, riemannType=1, dtType=1, CFL=0.5,
                                                  uBound=0.5 * np.sqrt(1.4), pBound=1.0)),
        "euler3d_p2_char": (box3d(3, 3, 3, (-2, -2, -2), (2, 2, 2), bcs=char6, perturb=0.1, seed=1), 1,
                            dict(order=2, dtType=1, CFL=0.5)),
        "euler3d_p3_periodic": (box3d(3, 3, 4, perturb=0.1, seed=2), 10,
                                dict(order=3, dtType=0, dt=1e-3)),
        "advection3d_p2": (box3d(3, 3, 3, (-2, -2, -2), (2, 2, 2), bcs=char6), 0,
                           dict(order=2, equation=0, dtType=1, CFL=0.3)),
        # viscous (LDG) cases
        "ns2d_p3_roe_ldg": (box2d(6, 6, -10, 10, -10, 10, perturb=0.1, seed=12), 1,
                            dict(order=3, riemannType=1, viscous=1, mu_inf=0.01, prandtl=0.72, fixVis=1,
                                 penFact=0.5, tau=1.0, dtType=1, CFL=0.3)),
        "ns2d_p4_sutherland": (box2d(5, 4, -10, 10, -10, 10, perturb=0.1, seed=13), 1,
                               dict(order=4, riemannType=0, viscous=1, mu_inf=0.02, prandtl=0.71, fixVis=0,
                                    c_sth=0.41, rt_inf=2.5, penFact=0.0, tau=1.0, dtType=0, dt=1e-3)),
        "tgv3d_p3": (box3d(3, 3, 3, (0, 0, 0), (2 * np.pi,) * 3, perturb=0.05, seed=14), 10,
                     dict(order=3, viscous=1, mu_inf=1.0 / 1600, prandtl=0.71, fixVis=1, penFact=0.0, tau=1.0,
                          dtType=0, dt=1e-3)),
        "ns3d_p2_penalty_walls": (box3d(3, 3, 3, (-2, -2, -1), (2, 2, 1),
                                        bcs={"zmin": "adiabatic_noslip", "zmax": "isothermal_noslip"},
                                        perturb=0.1, seed=15), 1,
                                  dict(order=2, viscous=1, mu_inf=0.01, prandtl=0.72, fixVis=1, penFact=0.3,
                                       tau=1.0, TWall=1.0, RGas=1.0 / 1.4, dtType=1, CFL=0.3)),
        "advdiff2d_p3": (box2d(6, 6, perturb=0.1, seed=16), 0,
                         dict(order=3, equation=0, viscous=1, diffD=0.05, penFact=0.2, tau=1.0, dtType=0,
                              dt=1e-3)),
    }


CASES = list(cases().keys())


@pytest.mark.parametrize("name", CASES)
def test_residual_fp64(oracle, name):
    mesh, ic, kw = cases()[name]
    a0 = 0.1 if ic == 10 else 0.0
    g, o = pair(oracle, mesh, ic, a0, **kw)
    g.calcResidual(0)
    o.calc_residual(0)
    assert relerr(g.get("U_fpts"), o.get("U_fpts")) < FP64_TOL
    assert relerr(g.get("divF_spts", 0), o.divF(0)) < FP64_TOL


@pytest.mark.parametrize("name", CASES)
def test_update_fp64(oracle, name):
    mesh, ic, kw = cases()[name]
    a0 = 0.1 if ic == 10 else 0.0
    g, o = pair(oracle, mesh, ic, a0, **kw)
    for _ in range(3):
        g.update(1)
        o.update(1)
        assert relerr(g.dt, o.dt) < FP64_TOL
    assert relerr(g.get("U_spts"), o.U()) < FP64_TOL
    assert abs(g.time - o.time) <= 1e-12 * max(o.time, 1e-300) + 1e-300


@pytest.mark.parametrize("timeType,dtType", [(0, 0), (0, 1), (2, 1), (5, 0), (4, 2)])
def test_rk_variants(oracle, timeType, dtType):
    from fr_learn_b200 import box2d

    mesh = box2d(6, 6, -10, 10, -10, 10, perturb=0.1, seed=3)
    g, o = pair(oracle, mesh, 1, order=3, riemannType=1, timeType=timeType, dtType=dtType, dt=1e-3, CFL=0.3)
    g.update(3)
    o.update(3)
    assert relerr(g.get("U_spts"), o.U()) < FP64_TOL


def test_unfused_entry_points_match_update(oracle):
    """calcResidual/timeStepA/timeStepB driven by hand (solver::update's body)
    equals the fused frg_update step."""
    from fr_learn_b200 import Solver, box2d

    mesh = box2d(6, 6, -10, 10, -10, 10, perturb=0.1, seed=4)
    kw = dict(order=4, riemannType=1, dtType=0, dt=2e-3)
    a, b = Solver(mesh, **kw), Solver(mesh, **kw)
    a.setInitialCondition(1)
    b.setInitialCondition(1)
    a.update(1)
    RKa, RKb = [0., .5, .5, 1.], [1 / 6, 1 / 3, 1 / 3, 1 / 6]
    b.copyUspts_U0()
    for s in range(3):
        b.calcResidual(s)
        b.timeStepA(s, RKa[s + 1])
    b.calcResidual(3)
    b.copyU0_Uspts()
    for s in range(4):
        b.timeStepB(s)
    assert relerr(a.get("U_spts"), b.get("U_spts")) < FP64_TOL


def test_residual_norm(oracle):
    from fr_learn_b200 import box2d

    mesh = box2d(6, 6, -10, 10, -10, 10, perturb=0.1, seed=5)
    g, o = pair(oracle, mesh, 1, order=3, riemannType=1)
    g.calcResidual(0)
    o.calc_residual(0)
    for t in (1, 2, 3):
        assert relerr(g.getNormResidual(t), o.residual_norm(t)) < FP64_TOL
    g.setMonitor(True)
    g.update(2)
    o.update(2)
    assert relerr(g.getNormResidual(2), o.residual_norm(2)) < FP64_TOL


MIXED_L2_TOL = 1e-6  # relative L2 of the mixed path against the FP64 oracle


def test_mixed_precision_bound(oracle):
    """Mixed mode (FP32 operators, fluxes, traces, metrics; FP64 Riemann
    pressure and RK accumulation) stays within 1e-6 relative L2 (1e-5 max
    norm) of the FP64 oracle over 20 RK4 steps of the perturbed-mesh vortex."""
    from fr_learn_b200 import FRG_MIXED, box2d

    mesh = box2d(8, 8, -10, 10, -10, 10, perturb=0.1, seed=7)
    g, o = pair(oracle, mesh, 1, order=4, riemannType=1, dtType=0, dt=5e-3, precision=FRG_MIXED)
    g.update(20)
    o.update(20)
    U, R = g.get("U_spts"), o.U()
    l2 = np.linalg.norm(U - R) / np.linalg.norm(R)
    assert l2 < MIXED_L2_TOL, l2
    assert relerr(U, R) < 1e-5


@pytest.mark.parametrize("name", CASES)
def test_mixed_precision_bound_every_case(oracle, name):
    """The mixed-mode bound on every parity case (2D / 3D, inviscid and
    viscous, periodic and walled): 5 RK4 steps within 1e-6 relative L2 of the
    FP64 oracle."""
    from fr_learn_b200 import FRG_MIXED

    mesh, ic, kw = cases()[name]
    a0 = 0.1 if ic == 10 else 0.0
    g, o = pair(oracle, mesh, ic, a0, precision=FRG_MIXED, **kw)
    g.update(5)
    o.update(5)
    U, R = g.get("U_spts"), o.U()
    l2 = np.linalg.norm(U - R) / np.linalg.norm(R)
    assert l2 < MIXED_L2_TOL, l2


def test_operators_match_oracle(oracle):
    from fr_learn_b200 import Solver, box2d, box3d

    for mesh, P in ((box2d(3, 3), 4), (box3d(3, 3, 3), 3)):
        g = Solver(mesh, order=P)
        o = oracle.Oracle(oracle.params(nDims=mesh.nDims, order=P), mesh)
        assert np.array_equal(g.operator(0), o.get("opp_spts_to_fpts").reshape(g.nFpts, g.nSpts))
        assert np.array_equal(g.operator(3), o.get("opp_correction").reshape(g.nSpts, g.nFpts))
        for d in range(mesh.nDims):
            assert np.array_equal(g.operator(1, d), o.get(f"opp_grad_spts{d}").reshape(g.nSpts, g.nSpts))
            assert np.array_equal(g.operator(2, d), o.get(f"opp_extrapolateFn{d}").reshape(g.nFpts, g.nSpts))


GOLDEN_INVISCID = ["euler_p2_char_fixeddt", "euler_p3_char_cfl", "euler_p2_charslip_cfl", "advection_p3",
                   "ns_p2_sutherland_ldg", "ns_p3_walls"]


@pytest.mark.parametrize("name", GOLDEN_INVISCID)
def test_gpu_vs_reference_golden(oracle, name):
    """The CUDA path against the reference's own outputs (tests/golden/)."""
    import os

    from fr_learn_b200 import Solver
    from test_oracle_golden import golden_case

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.npz"))
    mesh, kw, ic, nsteps = golden_case(oracle, g, name)
    pre = f"case/{name}/"
    kw.pop("nDims")
    s = Solver(mesh, **kw)
    s.setInitialCondition(ic)
    s.calcResidual(0)
    assert relerr(s.get("divF_spts", 0), g[pre + "r0_divF_spts"]) < FP64_TOL
    s2 = Solver(mesh, **kw)
    s2.setInitialCondition(ic)
    dts = []
    for _ in range(nsteps):
        s2.update(1)
        dts.append(s2.dt)
    assert relerr(s2.get("U_spts"), g[pre + "final_U_spts"]) < FP64_TOL
    assert relerr(dts, g[pre + "dt_hist"]) < FP64_TOL


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", ["periodic", "bump"])
def test_tma_kernel_matches_generic_kernel(monkeypatch, precision, case):
    """The TMA-tiled stage kernel of the fused update (2D) and the generic
    per-thread-load kernel agree: to FP64 rounding in FP64 mode; in mixed mode
    the TMA kernel multiplies by a stored FP32 1/detJ where the generic kernel
    divides by detJ, a difference at FP32 rounding level."""
    from fr_learn_b200 import Solver, box2d, bump2d

    if case == "periodic":
        mesh, ic, kw = box2d(9, 7, -10, 10, -10, 10, perturb=0.1, seed=21), 1, dict(order=4, riemannType=1, dtType=1)
    else:
        mesh, ic, kw = bump2d(12, 5), 0, dict(order=3, riemannType=1, dtType=1, uBound=0.5 * np.sqrt(1.4), pBound=1.0)
    monkeypatch.setenv("FRG_KERNEL", "generic")
    a = Solver(mesh, precision=precision, **kw)
    monkeypatch.delenv("FRG_KERNEL")
    b = Solver(mesh, precision=precision, **kw)
    for s in (a, b):
        s.setInitialCondition(ic)
        s.update(5)
    assert relerr(b.get("U_spts"), a.get("U_spts")) < (1e-13 if precision == 0 else 1e-6)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", ["periodic", "bump"])
def test_tile_variants_identical_and_autotune_restores(precision, case):
    """Every tile shape of the TMA stage kernel gives bit-identical results
    (the per-element arithmetic does not depend on the tile), and autotune
    leaves the solution, time and dt where they were."""
    from fr_learn_b200 import Solver, box2d, bump2d

    if case == "periodic":
        mesh, ic, kw = box2d(9, 7, -10, 10, -10, 10, perturb=0.1, seed=21), 1, dict(order=4, riemannType=1, dtType=1)
    else:
        mesh, ic, kw = bump2d(12, 5), 0, dict(order=3, riemannType=1, dtType=1, uBound=0.5 * np.sqrt(1.4), pBound=1.0)
    ref = None
    nvar = Solver(mesh, precision=precision, **kw).tile_variant_count()
    assert nvar == 12
    for v in range(nvar):
        s = Solver(mesh, precision=precision, **kw)
        s.set_tile_variant(v)
        s.setInitialCondition(ic)
        s.update(4)
        U = s.get("U_spts")
        if ref is None:
            ref = (U, s.time, s.dt)
        else:
            assert np.array_equal(U, ref[0]), f"variant {v}"
            assert s.time == ref[1] and s.dt == ref[2]
    s = Solver(mesh, precision=precision, **kw)
    s.setInitialCondition(ic)
    s.update(2)
    U2, t2, dt2 = s.get("U_spts"), s.time, s.dt
    v, ms = s.autotune(3)
    assert 0 <= v < nvar and ms[v] > 0
    assert np.array_equal(s.get("U_spts"), U2) and s.time == t2 and s.dt == dt2
    s.update(2)
    assert np.array_equal(s.get("U_spts"), ref[0])


@pytest.mark.parametrize("case", ["periodic_p4", "periodic_p2", "periodic_p5", "bump_p3"])
def test_persistent_variants_multi_tile_ragged_match_oracle(oracle, case):
    """The persistent stage kernels (ring and split variants, the ones the
    benchmark's autotuner picks) on meshes large enough that a block walks
    two or more tiles and the last tile is partial: the slot ring, the
    next-tile loads, the deferred per-tile dt and the short tile.  FP64: every
    variant bit-identical to the one-tile kernel and within 1e-12 of the
    oracle (state, dt of every step, time); mixed: within 1e-6 relative L2 of
    the FP64 oracle and every variant bit-identical to the one-tile kernel."""
    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver, box2d, bump2d

    # tiles of 16 (P = 2), 8 (P = 3, 4) or 4 (P = 5) elements in mixed
    # precision, half that in FP64; 592 persistent blocks on 148 SMs
    if case == "periodic_p4":  # 83 x 71 = 5,893 elements: 737 tiles of 8, 1,474 of 4
        mesh, ic = box2d(83, 71, -10, 10, -10, 10, perturb=0.1, seed=31), 1
        kw = dict(order=4, riemannType=1, dtType=1, CFL=0.5)
    elif case == "periodic_p2":  # 131 x 97 = 12,707 elements: 795 tiles of 16
        mesh, ic = box2d(131, 97, -10, 10, -10, 10, perturb=0.1, seed=32), 1
        kw = dict(order=2, riemannType=1, dtType=1, CFL=0.5)
    elif case == "periodic_p5":  # 5,893 elements: 1,474 tiles of 4
        mesh, ic = box2d(83, 71, -10, 10, -10, 10, perturb=0.05, seed=33), 1
        kw = dict(order=5, riemannType=1, dtType=1, CFL=0.3)
    else:  # 157 x 41 = 6,437 elements, boundaries on every side
        mesh, ic = bump2d(157, 41), 0
        kw = dict(order=3, riemannType=1, dtType=1, CFL=0.5, uBound=0.5 * np.sqrt(1.4), pBound=1.0)
    nsteps = 3
    o = oracle.Oracle(oracle.params(nDims=2, **kw), mesh)
    o.set_ic(ic)
    dts = []
    for _ in range(nsteps):
        o.update(1)
        dts.append(o.dt)
    R, t_o = o.U().copy(), o.time
    o.close()
    for prec in (FRG_FP64, FRG_MIXED):
        ref = None
        nvar = Solver(mesh, precision=prec, **kw).tile_variant_count()
        for v in range(nvar):
            s = Solver(mesh, precision=prec, **kw)
            s.set_tile_variant(v)
            s.setInitialCondition(ic)
            sdt = []
            for _ in range(nsteps):
                s.update(1)
                sdt.append(s.dt)
            U = s.get("U_spts")
            if ref is None:
                ref = (U, sdt, s.time)
                if prec == FRG_FP64:
                    assert relerr(sdt, dts) < FP64_TOL
                    assert relerr(U, R) < FP64_TOL
                    assert abs(s.time - t_o) <= 1e-12 * t_o
                else:
                    assert float(np.linalg.norm(U - R) / np.linalg.norm(R)) < 1e-6
            else:
                assert np.array_equal(U, ref[0]), f"precision {prec}, variant {v}"
                assert sdt == ref[1] and s.time == ref[2], f"precision {prec}, variant {v}"
            s.close()


def test_advection_config1_full_run(oracle):
    """The first benchmark configuration in full: 2D scalar advection of a
    Gaussian on the periodic square [-5,5]^2, 32 x 32 quads, P = 3, upwind
    flux, RK4, dt 1e-3, 1000 steps, FP64 against the oracle."""
    from fr_learn_b200 import box2d

    mesh = box2d(32, 32, -5.0, 5.0, -5.0, 5.0)
    g, o = pair(oracle, mesh, 0, order=3, equation=0, advectVx=1.0, advectVy=1.0, dt=1e-3)
    g.update(1000)
    o.update(1000)
    assert relerr(g.get("U_spts"), o.U()) < FP64_TOL
    assert abs(g.time - o.time) <= 1e-12 * o.time


def _visc3_cases():
    from fr_learn_b200 import box3d

    return {
        "tgv_periodic": (box3d(4, 3, 5, (0, 0, 0), (2 * np.pi,) * 3, perturb=0.05, seed=41), 10, 0.1,
                         dict(order=3, viscous=1, mu_inf=1.0 / 1600, prandtl=0.71, fixVis=1, penFact=0.0, tau=1.0,
                              dtType=0, dt=1e-3)),
        "walls_penalty": (box3d(3, 3, 3, (-2, -2, -1), (2, 2, 1),
                                bcs={"zmin": "adiabatic_noslip", "zmax": "isothermal_noslip"}, perturb=0.1,
                                seed=42), 1, 0.0,
                          dict(order=2, viscous=1, mu_inf=0.01, prandtl=0.72, fixVis=1, penFact=0.3, tau=1.0,
                               TWall=1.0, RGas=1.0 / 1.4, dtType=1, CFL=0.3)),
        "advdiff_char": (box3d(3, 4, 3, (-2, -2, -2), (2, 2, 2),
                               bcs={s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")},
                               perturb=0.1, seed=43), 0, 0.0,
                         dict(order=3, equation=0, viscous=1, diffD=0.05, penFact=0.2, tau=1.0, dtType=0,
                              dt=1e-3)),
        "sutherland_p4": (box3d(3, 3, 3, (0, 0, 0), (2 * np.pi,) * 3, perturb=0.05, seed=44), 10, 0.1,
                          dict(order=4, viscous=1, mu_inf=0.02, prandtl=0.71, fixVis=0, c_sth=0.41, rt_inf=2.5,
                               penFact=0.0, tau=1.0, dtType=1, CFL=0.3)),
    }


def test_visc3_tma_multi_tile_walls_match_oracle(oracle):
    """The 3D viscous TMA passes on a walled mesh large enough that the
    persistent stage pass walks two or three tiles per block (the next tile's
    gathers issued during the current one, the codes by tile parity) and the
    last tile holds one element: 11 x 11 x 13 hexes, P = 3, adiabatic and
    isothermal no-slip walls with the LDG penalty, CFL dt.  FP64 within 1e-12
    of the oracle (state, dt of every step, time); mixed within 1e-6 relative
    L2."""
    import os

    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver, box3d

    mesh = box3d(11, 11, 13, (-2, -2, -1), (2, 2, 1),
                 bcs={"zmin": "adiabatic_noslip", "zmax": "isothermal_noslip"}, perturb=0.1, seed=45)
    kw = dict(order=3, viscous=1, mu_inf=0.01, prandtl=0.72, fixVis=1, penFact=0.3, tau=1.0, TWall=1.0,
              RGas=1.0 / 1.4, dtType=1, CFL=0.3)
    nsteps = 3
    oracle.lib().orc_set_threads(os.cpu_count() or 1)
    o = oracle.Oracle(oracle.params(nDims=3, **kw), mesh)
    o.set_ic(1)
    dts = []
    for _ in range(nsteps):
        o.update(1)
        dts.append(o.dt)
    R, t_o = o.U().copy(), o.time
    o.close()
    for prec in (FRG_FP64, FRG_MIXED):
        g = Solver(mesh, precision=prec, **kw)
        g.setInitialCondition(1)
        gdt = []
        for _ in range(nsteps):
            g.update(1)
            gdt.append(g.dt)
        U = g.get("U_spts")
        if prec == FRG_FP64:
            assert relerr(gdt, dts) < FP64_TOL
            assert relerr(U, R) < FP64_TOL
            assert abs(g.time - t_o) <= 1e-12 * t_o
        else:
            assert float(np.linalg.norm(U - R) / np.linalg.norm(R)) < MIXED_L2_TOL
        g.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", list(_visc3_cases()))
def test_visc3_tma_kernels_match_generic_kernels(monkeypatch, precision, case):
    """The 3D viscous TMA passes of the fused update (the stage input landed
    in the padded point layout, the gradient recomputed in the stage pass,
    the boundary viscous flux formed in the gradient pass) agree with the
    generic per-thread-load kernels: to FP64 rounding (the TMA stage
    multiplies by a stored 1/detJ where the generic one divides), in mixed
    mode to FP32 rounding level."""
    from fr_learn_b200 import Solver

    mesh, ic, a0, kw = _visc3_cases()[case]
    monkeypatch.setenv("FRG_KERNEL", "generic")
    a = Solver(mesh, precision=precision, **kw)
    monkeypatch.delenv("FRG_KERNEL")
    b = Solver(mesh, precision=precision, **kw)
    for s in (a, b):
        s.setInitialCondition(ic, a0)
        s.update(5)
    assert relerr(b.get("U_spts"), a.get("U_spts")) < (1e-13 if precision == 0 else 1e-6)
    assert relerr(b.get("U_fpts"), a.get("U_fpts")) < (1e-13 if precision == 0 else 1e-6)
    if kw.get("dtType") == 1:
        assert relerr(b.dt, a.dt) < (1e-13 if precision == 0 else 1e-6)
