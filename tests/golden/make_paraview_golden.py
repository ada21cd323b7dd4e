"""Generates tests/golden/reference_paraview.npz from the FlurryPP reference itself.

Run where the reference sources are present, at $REFDIR (default /root/reference):

    python tests/golden/make_paraview_golden.py

For small 3D hexahedral cases the reference harness (oracle/_ref/refharness,
mode 'vtu') runs a few solver::update() steps, writes the ParaView / restart
file with writeParaview (src/output.cpp:103-391) and restarts a second solver
from it (solver::readRestartFile, src/solver.cpp:1420-1482).  Recorded per
case: the state, nodes, time and iteration the file was written from, the
file's text, and the state and time the reference's reader recovered.
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

OUT = os.path.join(HERE, "reference_paraview.npz")
CHAR6 = {s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}


def cases():
    m1 = box3d(2, 1, 1, (-2, -1, -1), (2, 1, 1), bcs=CHAR6, perturb=0.1, seed=3)
    m2 = box3d(1, 1, 1, (-1, -1, -1), (1, 1, 1), bcs=CHAR6, perturb=0.1, seed=4)
    return {
        "euler_p2": (m1, 3, dict(icType=1, order=2, dtType=0, dt=1e-3)),
        "euler_p3_cfl": (m2, 2, dict(icType=1, order=3, dtType=1, CFL=0.5)),
        "advection_p1": (m1, 2, dict(icType=0, order=1, equation=0, dtType=0, dt=1e-3)),
    }


def main():
    if not refcase.available():
        sys.exit("the reference sources are not present; nothing to do")
    refcase.build()
    out = {}
    for name, (mesh, nsteps, kw) in cases().items():
        r = refcase.run_vtu(mesh, nsteps=nsteps, **kw)
        pre = f"{name}/"
        for k in ("U_spts", "nodes", "time", "iter", "restart_U_spts", "restart_time"):
            out[pre + k] = r[k]
        out[pre + "vtu"] = np.frombuffer(r["vtu"].encode(), np.uint8)
        out[pre + "xv"] = mesh.xv
        out[pre + "order"] = np.array([kw["order"]])
        out[pre + "equation"] = np.array([kw.get("equation", 1)])
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
