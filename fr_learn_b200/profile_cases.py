"""Small, self-contained runs of single workloads for profiler captures
(`ncu ... python -m fr_learn_b200.profile_cases <case>`): each builds one
handle, runs a few steps or calls, synchronises and exits 0.

Cases:
  c2_mixed / c2_fp64   2D Euler vortex, 128 x 128 perturbed quads, P = 4,
                       Roe, RK4, CFL 0.5 (the benchmark workload), 4 steps
                       with the tile variant given as the second argument
  tgv_mixed / tgv_fp64 3D Navier-Stokes Taylor-Green, 32^3 hexes, P = 3,
                       2 RK4 steps
  opgemm               the tensor-core operator GEMMs (spts->fpts, grad_x,
                       correction) over the Taylor-Green arrays, 2 calls each
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def main(argv):
    sys.path.insert(0, ROOT)
    import bench  # the workload definitions

    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver

    case = argv[0] if argv else "c2_mixed"
    prec = FRG_FP64 if case.endswith("fp64") else FRG_MIXED
    if case.startswith("c2"):
        s = Solver(bench.c2_mesh(), precision=prec, **bench.c2_params())
        s.setInitialCondition(1)
        if len(argv) > 1:
            s.set_tile_variant(int(argv[1]))
        s.update(4)
        s.sync()
        print(case, "time", s.time)
    elif case.startswith("tgv"):
        s = Solver(bench.tgv_mesh(), precision=prec, **bench.tgv_params())
        s.setInitialCondition(10, bench.TGV_MA)
        s.update(2)
        s.sync()
        print(case, "time", s.time)
    elif case == "opgemm":
        import torch

        s = Solver(bench.tgv_mesh(), precision=FRG_MIXED, **bench.tgv_params())
        s.set_stream(torch.cuda.current_stream().cuda_stream)
        nV, nE, nS, nF = s.nFields, s.nEles, s.nSpts, s.nFpts
        ld = (nE + 31) // 32 * 32
        for which, (M, K) in ((0, (nF, nS)), (1, (nS, nS)), (3, (nS, nF))):
            X = torch.randn((nV, K, ld), dtype=torch.float32, device="cuda")
            Y = torch.empty((nV, M, ld), dtype=torch.float32, device="cuda")
            for _ in range(2):
                s.apply_operator(which, 0, X.data_ptr(), Y.data_ptr(), ld)
            s.sync()
            print(case, which, float(np.abs(Y.cpu().numpy()).max()))
        s.set_stream(None)
    else:
        raise SystemExit(f"unknown case {case!r}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
