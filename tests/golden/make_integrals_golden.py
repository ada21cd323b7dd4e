"""Generates tests/golden/reference_integrals.npz from the FlurryPP reference itself.

Run where the reference sources are present, at $REFDIR (default /root/reference):

    python tests/golden/make_integrals_golden.py

For small 3D hexahedral cases the reference harness (oracle/_ref/refharness,
mode 'integrals') runs a few solver::update() steps, one calcResidual(0), and
records the output integrals the reference computes from that state:
solver::computeWallForce (src/boundFace.cpp:330-378), solver::computeMassFlux
(src/boundFace.cpp:380-418) for errorNorm 0, 1, 2, and solver::integrateError
(src/solver.cpp:1507-1574, calcError src/funcs.cpp:1875-1979, testCase 1)
for errorNorm 0, 1, 2 at quadOrder 4.  Recorded per case: the mesh, the
effective parameters, the state and time after the steps, and the integrals.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import refcase  # noqa: E402
from fr_learn_b200 import box3d  # noqa: E402

OUT = os.path.join(HERE, "reference_integrals.npz")

CHAR_SLIP = {"xmin": "char", "xmax": "char", "ymin": "char", "ymax": "char", "zmin": "slip_wall", "zmax": "slip_wall"}
CHAR_WALLS = {"xmin": "char", "xmax": "char", "ymin": "char", "ymax": "char", "zmin": "adiabatic_noslip",
              "zmax": "isothermal_noslip"}
CHAR6 = {s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}


def cases():
    m1 = box3d(3, 3, 2, (-3, -3, -1), (3, 3, 1), bcs=CHAR_SLIP, perturb=0.1, seed=21)
    m2 = box3d(2, 3, 3, (-2, -2, -1), (2, 2, 1), bcs=CHAR_WALLS, perturb=0.1, seed=22)
    m3 = box3d(3, 3, 3, (-3, -3, -3), (3, 3, 3), bcs=CHAR6, perturb=0.1, seed=23)
    vis = dict(viscous=1, Re=50.0, MachBound=0.845, MachWall=0.0)
    q = dict(quadOrder=4)
    return {
        "euler_p2_vortex": (m1, 2, dict(icType=1, order=2, dtType=0, dt=1e-3, **q)),
        "euler_p3_freestream": (m1, 2, dict(icType=0, order=3, dtType=1, CFL=0.5, uBound=0.3, **q)),
        "ns_p2_walls": (m2, 2, dict(icType=1, order=2, dtType=1, CFL=0.3, fixVis=1, LDG_penFact=0.5, **vis, **q)),
        "ns_p3_sutherland_freestream": (m2, 1, dict(icType=0, order=3, dtType=1, CFL=0.3, fixVis=0, **vis, **q)),
        "advection_p3_gauss": (m3, 2, dict(icType=0, order=3, equation=0, dtType=0, dt=1e-3, **q)),
        "advection_p2_sine": (m3, 2, dict(icType=1, order=2, equation=0, dtType=0, dt=1e-3, **q)),
    }


def main():
    if not refcase.available():
        sys.exit("the reference sources are not present; nothing to do")
    refcase.build()
    out = {}
    for name, (mesh, nsteps, kw) in cases().items():
        r = refcase.run_integrals(mesh, nsteps=nsteps, **kw)
        pre = f"{name}/"
        out[pre + "xv"] = mesh.xv
        out[pre + "c2v"] = mesh.c2v
        out[pre + "bc"] = mesh.bc
        out[pre + "setup"] = np.array([kw.get("order"), kw.get("equation", 1), kw.get("viscous", 0),
                                       kw.get("icType", 0), kw["quadOrder"], nsteps], np.int64)
        for k in ["params", "U_spts", "time", "wall_force", "mass_flux_0", "mass_flux_1", "mass_flux_2",
                  "error_0", "error_1", "error_2"]:
            out[pre + k] = r[k]
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT) / 1024:.0f} kB")


if __name__ == "__main__":
    main()
