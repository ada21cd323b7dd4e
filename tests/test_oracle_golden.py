"""The oracle against the reference's own outputs (tests/golden/, made by
tests/golden/make_golden.py from the FlurryPP sources).  CPU only.

The oracle keeps the reference's arithmetic order, so on the same compiler it
agrees bit for bit; the bar here is 1e-13 relative so the check also holds
for other x86-64 toolchains."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import relerr

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "reference_golden.npz")
TOL = 1e-13


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _oracle_for_ops(oracle, d, P, v):
    from fr_learn_b200 import box2d, box3d

    mesh = box2d(3, 3) if d == 2 else box3d(3, 3, 3)
    return oracle.Oracle(oracle.params(nDims=d, order=P, vcjhScheme=v, viscous=1), mesh)


@pytest.mark.parametrize("d,P,v", [(2, P, 0) for P in range(1, 6)] + [(3, P, 0) for P in range(1, 5)]
                         + [(2, 3, 1), (2, 3, 2), (3, 3, 1), (3, 3, 2)])
def test_operators(oracle, golden, d, P, v):
    o = _oracle_for_ops(oracle, d, P, v)
    pre = f"ops/{d}d_p{P}_v{v}/"
    nS, nF = o.nS, o.nF
    assert np.array_equal(o.get("opp_spts_to_fpts").reshape(nF, nS), golden[pre + "spts_to_fpts"])
    assert np.array_equal(o.get("opp_correction").reshape(nS, nF), golden[pre + "correction"])
    for k in range(d):
        assert np.array_equal(o.get(f"opp_grad_spts{k}").reshape(nS, nS), golden[pre + f"grad_spts_{k}"])
        assert np.array_equal(o.get(f"opp_extrapolateFn{k}").reshape(nF, nS), golden[pre + f"extrapolateFn_{k}"])
        assert np.array_equal(o.get(f"opp_correctU{k}").reshape(nS, nF), golden[pre + f"correctU_{k}"])


def _kat_params(oracle, d, **kw):
    base = dict(nDims=d, equation=1, gamma=1.4, rhoBound=1.0, uBound=0.5 * np.sqrt(1.4), vBound=0.1,
                wBound=-0.05 if d == 3 else 0.0, pBound=1.0, mu_inf=1.0 / 1600.0, prandtl=0.71, fixVis=1,
                c_sth=0.41, rt_inf=2.5, penFact=0.3, tau=1.0, viscous=1)
    base.update(kw)
    return oracle.params(**base)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("fix", [0, 1])
def test_kat_point_fluxes(oracle, golden, d, fix):
    L = oracle.lib()
    L.orc_point_flux.argtypes = [C.POINTER(oracle.OrcParams)] + [C.c_void_p] * 4
    p = _kat_params(oracle, d, fixVis=fix)
    s = f"_{d}d_fix{fix}"
    U, G = golden["kat/flux_U" + s], golden["kat/flux_gradU" + s]
    nV = d + 2
    Fi = np.zeros((len(U), d, nV))
    Fv = np.zeros((len(U), d, nV))
    for i in range(len(U)):
        u = np.ascontiguousarray(U[i])
        g = np.ascontiguousarray(G[i])
        a, b = np.zeros((d, nV)), np.zeros((d, nV))
        L.orc_point_flux(C.byref(p), _ptr(u), _ptr(g), _ptr(a), _ptr(b))
        Fi[i], Fv[i] = a, b
    assert relerr(Fi, golden["kat/flux_inv" + s]) < TOL
    assert relerr(Fv, golden["kat/flux_vis" + s]) < TOL


@pytest.mark.parametrize("d", [2, 3])
def test_kat_riemann(oracle, golden, d):
    L = oracle.lib()
    P = C.POINTER(oracle.OrcParams)
    L.orc_point_rusanov.argtypes = [P] + [C.c_void_p] * 4
    L.orc_point_rusanov.restype = C.c_double
    L.orc_point_roe.argtypes = [P] + [C.c_void_p] * 4
    L.orc_point_ldg_uc.argtypes = [P] + [C.c_void_p] * 4
    p = _kat_params(oracle, d)
    s = f"_{d}d"
    UL, UR, N = golden["kat/face_UL" + s], golden["kat/face_UR" + s], golden["kat/face_norm" + s]
    nV = d + 2
    Fr, W, Fro, UC = np.zeros((len(UL), nV)), np.zeros(len(UL)), np.zeros((len(UL), nV)), np.zeros((len(UL), nV))
    for i in range(len(UL)):
        ul, ur, n = (np.ascontiguousarray(x[i]) for x in (UL, UR, N))
        f = np.zeros(nV)
        W[i] = L.orc_point_rusanov(C.byref(p), _ptr(ul), _ptr(ur), _ptr(n), _ptr(f))
        Fr[i] = f
        c = np.zeros(nV)
        L.orc_point_ldg_uc(C.byref(p), _ptr(ul), _ptr(ur), _ptr(n), _ptr(c))
        UC[i] = c
        if d == 2:
            g = np.zeros(nV)
            L.orc_point_roe(C.byref(p), _ptr(ul), _ptr(ur), _ptr(n), _ptr(g))
            Fro[i] = g
    assert relerr(Fr, golden["kat/face_rusanov" + s]) < TOL
    assert relerr(W, golden["kat/face_rusanov_wavesp" + s]) < TOL
    assert relerr(UC, golden["kat/face_ldgUC" + s]) < TOL
    if d == 2:
        assert relerr(Fro, golden["kat/face_roe" + s]) < TOL


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("bc", ["char", "slip_wall", "sup_in", "sup_out"])
@pytest.mark.parametrize("regime", ["sub", "sup"])
def test_kat_boundary_states(oracle, golden, d, bc, regime):
    from fr_learn_b200.mesh import BC

    L = oracle.lib()
    L.orc_point_bc.argtypes = [C.POINTER(oracle.OrcParams), C.c_int] + [C.c_void_p] * 3
    s = f"_{d}d_{bc}_{regime}"
    rho, u, v, pb = golden["kat/bc_bound" + s]
    p = _kat_params(oracle, d, rhoBound=rho, uBound=u, vBound=v, pBound=pb, viscous=0)
    UL, N = golden["kat/bc_UL" + s], golden["kat/bc_norm" + s]
    UR = np.zeros_like(UL)
    for i in range(len(UL)):
        ul, n = np.ascontiguousarray(UL[i]), np.ascontiguousarray(N[i])
        r = np.zeros(d + 2)
        L.orc_point_bc(C.byref(p), BC[bc], _ptr(ul), _ptr(n), _ptr(r))
        UR[i] = r
    assert relerr(UR, golden["kat/bc_UR" + s]) < TOL


@pytest.mark.parametrize("d", [2, 3])
def test_kat_lax_friedrichs(oracle, golden, d):
    L = oracle.lib()
    L.orc_point_lf.argtypes = [C.POINTER(oracle.OrcParams), C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    L.orc_point_lf.restype = C.c_double
    p = oracle.params(nDims=d, equation=0, advectVx=1.0, advectVy=1.0, advectVz=0.5 if d == 3 else 0.0)
    s = f"_{d}d"
    uL, uR, N = golden["kat/lf_uL" + s], golden["kat/lf_uR" + s], golden["kat/lf_norm" + s]
    Fn, W = np.zeros(len(uL)), np.zeros(len(uL))
    for i in range(len(uL)):
        f = np.zeros(1)
        W[i] = L.orc_point_lf(C.byref(p), float(uL[i]), float(uR[i]), _ptr(np.ascontiguousarray(N[i])), _ptr(f))
        Fn[i] = f[0]
    assert relerr(Fn, golden["kat/lf_Fn" + s]) < TOL
    assert relerr(W, golden["kat/lf_wavesp" + s]) < TOL


CASES = ["euler_p2_char_fixeddt", "euler_p3_char_cfl", "euler_p2_charslip_cfl", "ns_p2_sutherland_ldg",
         "ns_p3_walls", "advection_p3"]
PNAMES = ["gamma", "rhoBound", "uBound", "vBound", "wBound", "pBound", "mu_inf", "prandtl", "c_sth", "rt_inf",
          "fixVis", "penFact", "tau", "TWall", "RGas", "uWall", "vWall", "wWall", "dt", "CFL"]


def golden_case(oracle, golden, name):
    """The golden mesh and the oracle set up with the reference's effective parameters."""
    from fr_learn_b200.mesh import Mesh

    pre = f"case/{name}/"
    mesh = Mesh(3, golden[pre + "xv"], golden[pre + "c2v"], golden[pre + "bc"])
    order, equation, viscous, dtType, icType, nsteps = (int(x) for x in golden[pre + "setup"])
    prm = dict(zip(PNAMES, golden[pre + "params"].tolist()))
    prm["fixVis"] = int(prm["fixVis"])
    kw = dict(nDims=3, order=order, equation=equation, viscous=viscous, dtType=dtType, riemannType=0, **prm)
    return mesh, kw, icType, nsteps


@pytest.mark.parametrize("name", CASES)
def test_cases_residual_and_steps(oracle, golden, name):
    mesh, kw, ic, nsteps = golden_case(oracle, golden, name)
    pre = f"case/{name}/"
    o = oracle.Oracle(oracle.params(**kw), mesh)
    o.set_ic(ic)
    assert relerr(o.get("pos_spts"), golden[pre + "pos_spts"]) < TOL
    assert relerr(o.get("detJac_spts"), golden[pre + "detJac_spts"]) < TOL
    assert sorted(map(tuple, o.faces().tolist())) == sorted(map(tuple, golden[pre + "faces"].tolist()))
    o.calc_residual(0)
    assert relerr(o.get("U_fpts"), golden[pre + "r0_U_fpts"]) < TOL
    assert relerr(o.get("Fn_fpts"), golden[pre + "r0_Fn_fpts"]) < TOL
    assert relerr(o.get("divF_spts0"), golden[pre + "r0_divF_spts"]) < TOL
    if kw["viscous"]:
        assert relerr(o.get("dU_spts"), golden[pre + "r0_dU_spts"]) < TOL
        assert relerr(o.get("dUc_fpts"), golden[pre + "r0_dUc_fpts"]) < TOL
    o2 = oracle.Oracle(oracle.params(**kw), mesh)
    o2.set_ic(ic)
    dts, res = [], []
    for _ in range(nsteps):
        o2.update(1)
        dts.append(o2.dt)
        res.append(o2.residual_norm(2))
    assert relerr(o2.get("U_spts"), golden[pre + "final_U_spts"]) < TOL
    assert relerr(dts, golden[pre + "dt_hist"]) < TOL
    assert relerr(res, golden[pre + "res_hist"]) < 1e-12
    assert abs(o2.time - float(golden[pre + "final_time"][0])) <= 1e-13 * max(1.0, o2.time)
