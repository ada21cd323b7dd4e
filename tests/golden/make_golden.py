"""Generates tests/golden/reference_golden.npz from the FlurryPP reference itself.

Run where the reference sources are present, at $REFDIR (default /root/reference):

    python tests/golden/make_golden.py

It builds oracle/_ref/refharness (oracle/Makefile: the reference's own
sources + a plain-C cblas_dgemm shim) and records:

* ops/   operator matrices of oper::setupOperators for QUAD (P=1..5) and HEX
         (P=1..4), DG correction, plus SD / HU at P=3;
* kat/   pointwise known answers: inviscidFlux / viscousFlux (2D, 3D,
         Sutherland on/off), Rusanov, 2D Roe, Lax-Friedrichs, the LDG common
         solution and boundFace::applyBCs for char / slip / sup_in / sup_out;
* case/  3D hexahedral cases run by solver::setup / calcResidual / update:
         the mesh, the effective parameters, one residual with its
         intermediate arrays and a few time steps (final state, dt history,
         L2 residual norms).

The fixture is small (a few hundred kB compressed) and is what the CPU tests
pin the oracle to, on machines without the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import refcase  # noqa: E402
from fr_learn_b200 import box3d  # noqa: E402

OUT = os.path.join(HERE, "reference_golden.npz")

CHAR6 = {s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
CHAR_SLIP = {"xmin": "char", "xmax": "char", "ymin": "char", "ymax": "char", "zmin": "slip_wall", "zmax": "slip_wall"}
CHAR_WALLS = {"xmin": "char", "xmax": "char", "ymin": "char", "ymax": "char", "zmin": "adiabatic_noslip",
              "zmax": "isothermal_noslip"}


def cases():
    m1 = box3d(3, 3, 3, (-2, -2, -2), (2, 2, 2), bcs=CHAR6, perturb=0.1, seed=1)
    m2 = box3d(3, 2, 3, (-2, -2, -1), (2, 2, 1), bcs=CHAR_SLIP, perturb=0.1, seed=2)
    m3 = box3d(2, 3, 3, (-2, -2, -1), (2, 2, 1), bcs=CHAR_WALLS, perturb=0.1, seed=3)
    vis = dict(viscous=1, Re=50.0, MachBound=0.845, MachWall=0.0)
    return {
        "euler_p2_char_fixeddt": (m1, 3, dict(icType=1, order=2, dtType=0, dt=1e-3)),
        "euler_p3_char_cfl": (m1, 3, dict(icType=1, order=3, dtType=1, CFL=0.5)),
        "euler_p2_charslip_cfl": (m2, 3, dict(icType=1, order=2, dtType=1, CFL=0.5)),
        "ns_p2_sutherland_ldg": (m2, 3, dict(icType=1, order=2, dtType=1, CFL=0.3, fixVis=0, LDG_penFact=0.5,
                                             LDG_tau=1.0, **vis)),
        "ns_p3_walls": (m3, 2, dict(icType=1, order=3, dtType=1, CFL=0.3, fixVis=1, **vis)),
        "advection_p3": (m1, 2, dict(icType=0, order=3, equation=0, dtType=0, dt=1e-3)),
    }


# effective parameters dumped by the harness, in order
PARAM_NAMES = ["gamma", "rhoBound", "uBound", "vBound", "wBound", "pBound", "mu_inf", "prandtl", "c_sth",
               "rt_inf", "fixVis", "penFact", "tau", "TWall", "RGas", "uWall", "vWall", "wWall", "dt", "CFL"]


def main():
    if not refcase.available():
        sys.exit("the reference sources are not present; nothing to do")
    refcase.build()
    out = {}
    for d, orders in ((2, range(1, 6)), (3, range(1, 5))):
        for P in orders:
            for v in ([0, 1, 2] if P == 3 else [0]):
                r = refcase.run_ops(d, P, v)
                for k, a in r.items():
                    out[f"ops/{d}d_p{P}_v{v}/{k}"] = a
    for k, a in refcase.run_kat().items():
        out[f"kat/{k}"] = a
    for name, (mesh, nsteps, kw) in cases().items():
        r = refcase.run_case(mesh, nsteps=nsteps, **kw)
        pre = f"case/{name}/"
        out[pre + "xv"] = mesh.xv
        out[pre + "c2v"] = mesh.c2v
        out[pre + "bc"] = mesh.bc
        out[pre + "params"] = r["params"]
        out[pre + "setup"] = np.array([kw.get("order"), kw.get("equation", 1), kw.get("viscous", 0),
                                       kw.get("dtType", 0), kw.get("icType", 0), nsteps], np.int64)
        keep = ["pos_spts", "detJac_spts", "dA_fpts", "faces", "r0_U_fpts", "r0_Fn_fpts", "r0_divF_spts",
                "final_U_spts", "dt_hist", "res_hist", "final_time"]
        if kw.get("viscous"):
            keep += ["r0_dU_spts", "r0_dUc_fpts"]
        for k in keep:
            out[pre + k] = r[k]
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT) / 1024:.0f} kB")


if __name__ == "__main__":
    main()
