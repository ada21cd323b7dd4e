"""Benchmark of the FR residual + RK4 path: DOF-updates/s on B200.

Workload (default): 2D Euler isentropic vortex (strength 5, centred at the
origin, freestream rho = p = 1, u = (1,1)) on the periodic square
[-10,10]^2, 128 x 128 linear quads with vertices perturbed by up to 10% of
the spacing (seed 0), order P = 4 (Gauss points, DG correction), gamma 1.4,
Roe flux, RK44, global CFL 0.5.  Synthetic inputs; no dataset involved.

One step = one full RK4 step (dt reduction + 4 fused stage kernels) over all
16384 elements; DOF = nEles * nSpts * nFields = 1,638,400.  `value` is the
mixed-precision path; the FP64 path is reported beside it.

Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events
on the solver's stream; L2 is flushed (a 512 MiB write) before every step,
outside the events.  Multi-GPU: independent replicas, one per rank
(`scaling: weak`), time = max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, ORDER = 128, 4
METRIC = "DOF-updates/s on 1 B200: mixed vs FP64 at stated error; adjoint/forward time"
UNIT = "DOF-updates/s"
WORKLOAD = "euler2d_isentropic_vortex_periodic_128x128_P4_roe_rk44_cfl0.5"
FALLBACK_HBM_GBS = 6650.0


def c2_mesh():
    from fr_learn_b200 import box2d

    return box2d(NX, NX, -10.0, 10.0, -10.0, 10.0, perturb=0.1, seed=0)


def c2_params(**kw):
    d = dict(order=ORDER, equation=1, riemannType=1, timeType=4, dtType=1, CFL=0.5, gamma=1.4,
             rhoBound=1.0, uBound=1.0, vBound=1.0, pBound=1.0)
    d.update(kw)
    return d


def bytes_per_dof_update(nDims, P, nV, s, g, viscous=False):
    """Algorithmic bytes per DOF-update (4 RK stages), the per-element model:
    nS*nV*(2s+24) + nS*(d^2+1)*g + nF*(d+1)*g + 4*nF*nV*s + 4*nF per stage,
    plus (2+2d)*nF*nV*s for a viscous stage (the common-solution and gradient
    traces)."""
    n1 = P + 1
    nS = n1 ** nDims
    nF = 2 * nDims * n1 ** (nDims - 1)
    per_stage = nS * nV * (2 * s + 24) + nS * (nDims * nDims + 1) * g + nF * (nDims + 1) * g + 4 * nF * nV * s + 4 * nF
    if viscous:
        per_stage += (2 + 2 * nDims) * nF * nV * s
    return 4 * per_stage / (nS * nV)


def max_over_ranks(x, world, device=None):
    """Maximum of a per-rank time over all ranks (every rank calls this in
    the same order); a no-op on one rank."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(n_ranks, dof, ms_per_step):
    """Whole-job DOF-updates/s: every rank advances `dof` unknowns per step
    (replicas), the job takes the slowest rank's time."""
    return n_ranks * dof / (ms_per_step * 1e-3)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons of one GPU, sampled through NVML by a
    background thread every ~10 ms from before the warm-up until after the
    timed region.  `mark(True/False)` brackets the timed region; the summary
    uses the samples taken inside it or, for a region shorter than the
    sampling interval, the samples on either side of it."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4))

    def __init__(self, device_index):
        self.idx = device_index
        self.samples = []  # (time, sm MHz, reason bits)
        self.windows = []
        self.max_mhz = None
        self.error = None

    def _handle(self, nv):
        import torch

        try:
            uuid = str(torch.cuda.get_device_properties(self.idx).uuid)
            return nv.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:  # noqa: BLE001 -- fall back to the visible index
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x for x in vis.split(",") if x.strip()]
            phys = int(ids[self.idx]) if self.idx < len(ids) and ids[self.idx].strip().isdigit() else self.idx
            return nv.nvmlDeviceGetHandleByIndex(phys)

    def __enter__(self):
        import threading

        self._stop = threading.Event()
        try:
            import pynvml as nv

            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception as e:  # noqa: BLE001
            self.error = f"NVML unavailable: {e}"
            return self

        def loop():
            while not self._stop.is_set():
                try:
                    mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((time.perf_counter(), float(mhz), int(bits)))
                except Exception as e:  # noqa: BLE001
                    self.error = str(e)
                    return
                self._stop.wait(0.01)

        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()
        time.sleep(0.05)
        return self

    def mark(self, start):
        if start:
            self.windows.append([time.perf_counter(), None])
        else:
            self.windows[-1][1] = time.perf_counter()

    def __exit__(self, *a):
        self._stop.set()
        if getattr(self, "_thread", None) is not None:
            self._thread.join(timeout=2)

    def summary(self):
        inside, near = [], []
        for t0, t1 in self.windows:
            if t1 is None:
                continue
            w = [x for x in self.samples if t0 <= x[0] <= t1]
            if w:
                inside += w
            else:
                before = [x for x in self.samples if x[0] < t0][-1:]
                after = [x for x in self.samples if x[0] > t1][:1]
                near += before + after
        use = inside or near
        reasons = sorted({n for _, _, bits in use for n, b in self.REASONS if bits & b})
        out = {"sm_mhz": statistics.median(x[1] for x in use) if use else None, "sm_max_mhz": self.max_mhz,
               "reasons": reasons, "samples": len(use),
               "source": "NVML every ~10 ms, " + ("inside the timed regions" if inside else
                                                   "nearest samples around timed regions shorter than the interval")}
        if self.error:
            out["error"] = self.error
        return out


def run_gpu(args, rank, world, local_rank):
    import torch

    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    mesh = c2_mesh()
    res = {}
    solvers = {}
    for name, prec in (("mixed", FRG_MIXED), ("fp64", FRG_FP64)):
        s = Solver(mesh, precision=prec, **c2_params())
        s.set_stream(stream.cuda_stream)
        s.setInitialCondition(1)
        # tile shape of the fused stage kernel, timed on this mesh (the
        # solution is restored afterwards), or the one given
        if args.tile_variants:
            v = int(args.tile_variants.split(",")[0 if name == "mixed" else 1])
            s.set_tile_variant(v)
            res.setdefault("tile_variant", {})[name] = v
        else:
            with torch.cuda.stream(stream):
                res.setdefault("tile_variant", {})[name] = int(s.autotune(10)[0])
        solvers[name] = s
    dof = solvers["mixed"].nEles * solvers["mixed"].nSpts * solvers["mixed"].nFields
    sampler = ClockSampler(local_rank)
    with sampler:
        for name, s in solvers.items():
            with torch.cuda.stream(stream):
                for _ in range(args.warmup):
                    flush.fill_(1)
                    s.update(1)
                stream.synchronize()
                if world > 1:
                    torch.distributed.barrier()
                torch.cuda.synchronize()
                launches0 = s.launch_count()
                ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                      for _ in range(args.steps)]
                sampler.mark(True)
                # an NVTX range names the timed region (profiler launch lists:
                # ncu --nvtx --nvtx-include "timed_<precision>/")
                torch.cuda.nvtx.range_push(f"timed_{name}")
                t_wall = time.perf_counter()
                for k in range(args.steps):
                    flush.fill_(k & 0xFF)
                    ev[k][0].record(stream)
                    s.update(1)
                    ev[k][1].record(stream)
                stream.synchronize()
                t_wall = time.perf_counter() - t_wall
                torch.cuda.nvtx.range_pop()
                sampler.mark(False)
                if world > 1:
                    torch.distributed.barrier()
                torch.cuda.synchronize()
                ms = sum(a.elapsed_time(b) for a, b in ev)
                launches = s.launch_count() - launches0
            ms = max_over_ranks(ms, world, dev)
            res[name] = {"ms_total": ms, "ms_per_step": ms / args.steps, "launches": launches, "wall_s": t_wall}
    clocks = sampler.summary()
    # the same steps back to back with no flush between them: the ~90 MB
    # working set stays in the 126 MB L2 from one step to the next, as in a
    # long run (reported beside the headline, not as it)
    for name, s in solvers.items():
        n_warm = max(20, min(args.steps, 500))
        with torch.cuda.stream(stream):
            s.update(3)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s.update(n_warm)
            b.record(stream)
            stream.synchronize()
        res[name]["l2_resident_ms_per_step"] = max_over_ranks(a.elapsed_time(b), world, dev) / n_warm
    # accuracy of the mixed path against the FP64 path after the same steps
    # (the FP64 path matches the FP64 oracle to 1e-12, see tests/)
    Um, Ud = solvers["mixed"].get("U_spts"), solvers["fp64"].get("U_spts")
    err_l2 = float(np.linalg.norm(Um - Ud) / np.linalg.norm(Ud))
    err_linf = float(np.abs(Um - Ud).max() / np.abs(Ud).max())
    # error of the FP64 density against the exact convected vortex
    # (calcError, src/funcs.cpp:1902-1950, on the [-10,10]^2 period)
    t_phys = solvers["fp64"].time
    pos = solvers["fp64"].get("pos_spts")
    x = np.mod(pos[..., 0] - t_phys + 10.0, 20.0) - 10.0
    y = np.mod(pos[..., 1] - t_phys + 10.0, 20.0) - 10.0
    g = 1.4
    f = 1.0 - (x * x + y * y)
    rho_ex = np.maximum((1.0 - 25.0 * (g - 1.0) / (8.0 * g * np.pi ** 2) * np.exp(f)) ** (1.0 / (g - 1.0)), 1e-10)
    rho_err = float(np.linalg.norm(Ud[..., 0] - rho_ex) / np.linalg.norm(rho_ex))

    # per-launch kernel durations (same kernels, launched without the graph)
    stage_ms = {}
    for name, s in solvers.items():
        with torch.cuda.stream(stream):
            stage_ms[name] = s.time_stages(max(3, min(50, args.steps)), flush.data_ptr(), flush.numel()).tolist()

    # end to end through the C ABI with host buffers: each step uploads the
    # state from pinned memory, runs update(), downloads the state
    s = solvers["mixed"]
    Uh = torch.empty((s.nSpts, s.nEles, s.nFields), dtype=torch.float64, pin_memory=True)
    Uh.numpy()[...] = s.get("U_spts")
    n_e2e = max(3, min(args.steps, 200))
    with torch.cuda.stream(stream):
        for _ in range(2):
            s.update_host(Uh.numpy(), 1)
        stream.synchronize()
        e2e_ms = 0.0
        for k in range(n_e2e):
            flush.fill_(k & 0xFF)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s.update_host(Uh.numpy(), 1)
            b.record(stream)
            b.synchronize()
            e2e_ms += a.elapsed_time(b)
    e2e_ms = max_over_ranks(e2e_ms, world, dev)
    # the host link's own bound for that step: one pinned H2D and one D2H
    # copy of the state, nothing else
    Ud = torch.empty(Uh.shape, dtype=torch.float64, device=dev)
    with torch.cuda.stream(stream):
        for _ in range(2):
            Ud.copy_(Uh, non_blocking=True)
            Uh.copy_(Ud, non_blocking=True)
        stream.synchronize()
        cp_ms = 0.0
        for k in range(n_e2e):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            Ud.copy_(Uh, non_blocking=True)
            Uh.copy_(Ud, non_blocking=True)
            b.record(stream)
            b.synchronize()
            cp_ms += a.elapsed_time(b)
    copy_ms = max_over_ranks(cp_ms, world, dev) / n_e2e
    state_bytes = s.nSpts * s.nEles * s.nFields * 8
    for sv in solvers.values():
        sv.set_stream(None)
    res["adjoint"] = run_adjoint_bump(stream)
    res["ensemble"] = run_ensemble(stream)
    res["tgv"] = run_tgv(stream, flush)
    res["tgv"]["kinetic_energy_vs_fp64_oracle"] = run_tgv_oracle(stream)
    res["c1"] = run_advection_c1(stream)
    res["scale"] = run_scale(stream, flush)
    res["opgemm"] = run_operator_gemm(stream, flush)
    return dof, res, stage_ms, clocks, (err_l2, err_linf, rho_err, t_phys), (e2e_ms / n_e2e, state_bytes, copy_ms)


def run_adjoint_bump(stream, nsteps=500, every=25):
    """Adjoint workload: 2D Euler channel over a Gaussian bump (96x32
    quadratic quads clustered to the wall, P=3, Roe, char inlet/outlet at
    Mach 0.5, slip lower wall, symmetry top), freestream initial state, RK4
    with the CFL-0.5 dt of the first step held fixed, 500 steps; J = pressure
    integral over the lower wall at the final time; gradients dJ/dU_0 and
    dJ/dMach by the reverse RK sweep with checkpoints every 25 steps.
    Returns forward and adjoint times per step (CUDA events)."""
    import torch

    from fr_learn_b200 import Solver, bump2d

    g = 1.4
    c = np.sqrt(g)
    M = 0.5
    mesh = bump2d(96, 32, bc_top="symmetry")
    kw = dict(order=3, riemannType=1, timeType=4, uBound=M * c, pBound=1.0, rhoBound=1.0)
    s0 = Solver(mesh, dtType=1, CFL=0.5, **kw)
    s0.setInitialCondition(0)
    s0.update(1)
    dt = s0.dt

    def make(Mach):
        s = Solver(mesh, dtType=0, dt=dt, **dict(kw, uBound=Mach * c))
        s.set_stream(stream.cuda_stream)
        s.setInitialCondition(0)
        return s

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            r = fn()
            b.record(stream)
            b.synchronize()
        return a.elapsed_time(b), r

    s = make(M)
    s.update(3)  # warm-up (graphs, kernels)
    s.setInitialCondition(0)
    fwd_ms, _ = timed(lambda: s.update(nsteps))
    theta = np.array([0.0, c, 0.0, 0.0, 0.0])
    # one untimed forward + reverse sweep: the segment recomputation and
    # reversal graphs are captured on first use (set-up, like the forward's
    # warm-up steps)
    s.setInitialCondition(0)
    s.adjoint_forward(nsteps, every)
    s.objective("wall_pressure")
    s.adjoint_backward(None, theta)
    s.setInitialCondition(0)
    U0 = s.get("U_spts")
    rec_ms, _ = timed(lambda: s.adjoint_forward(nsteps, every))
    J, _ = s.objective("wall_pressure")
    adj_ms, (lam0, tbar) = timed(lambda: s.adjoint_backward(None, theta))
    # the same gradient with every stage state kept by the forward run
    # (nsteps x 4 states in HBM; the reverse sweep recomputes nothing), after
    # one untimed run that allocates the stage store and captures the graphs
    s.setInitialCondition(0)
    s.adjoint_forward(nsteps, 0)
    s.objective("wall_pressure")
    s.adjoint_backward(None, theta)
    s.setInitialCondition(0)
    keep_fwd_ms, _ = timed(lambda: s.adjoint_forward(nsteps, 0))
    s.objective("wall_pressure")
    keep_ms, (lam0k, tbark) = timed(lambda: s.adjoint_backward(None, theta))
    rho = U0[..., 0]
    dU = np.zeros_like(U0)
    dU[..., 1] = rho * c
    dU[..., 3] = U0[..., 1] * c
    dJdM = float(np.sum(lam0 * dU)) + tbar
    # central difference of the forward solver over the Mach number
    eps = 1e-6
    Jpm = []
    for sg in (1, -1):
        s2 = make(M + sg * eps)
        s2.update(nsteps)
        Jpm.append(s2.objective("wall_pressure")[0])
        s2.set_stream(None)
    s.set_stream(None)
    fd = (Jpm[0] - Jpm[1]) / (2 * eps)
    return {"workload": "euler2d_bump_channel_96x32_q9_P3_roe_char_slip_M0.5_rk44_500steps",
            "steps": nsteps, "checkpoint_every": every, "dt": dt, "dof": s.nEles * s.nSpts * s.nFields,
            "forward_ms_per_step": fwd_ms / nsteps, "forward_with_checkpoints_ms_per_step": rec_ms / nsteps,
            "adjoint_ms_per_step": adj_ms / nsteps, "adjoint_over_forward": adj_ms / fwd_ms,
            "keep_all_stages": {"forward_ms_per_step": keep_fwd_ms / nsteps,
                                "adjoint_ms_per_step": keep_ms / nsteps, "adjoint_over_forward": keep_ms / fwd_ms,
                                "max_rel_diff_vs_checkpointed": float(np.abs(lam0k - lam0).max()
                                                                      / np.abs(lam0).max())},
            "J_wall_pressure": J, "dJ_dMach": dJdM, "dJ_dMach_central_difference": fd,
            "dJ_dMach_rel_diff": abs(dJdM - fd) / abs(fd)}


def ensemble_cases(n=256, seed=2024):
    """The batched workload: n independent 2D Euler isentropic-vortex cases on
    periodic [-10,10]^2 squares of side x side perturbed quads, side uniform
    in {16,24,...,96}, order P uniform in {2,3,4,5}, vortex strength uniform
    in [1,5], freestream Mach uniform in [0.1,0.6] along (1,1) (rho = p = 1),
    all drawn from one seeded generator."""
    rng = np.random.default_rng(seed)
    sides = np.arange(16, 97, 8)
    out = []
    for c in range(n):
        out.append(dict(side=int(rng.choice(sides)), P=int(rng.integers(2, 6)), eps=float(rng.uniform(1, 5)),
                        mach=float(rng.uniform(0.1, 0.6)), seed=c))
    return out


def vortex_state(pos, eps, mach, gamma=1.4):
    """Isentropic vortex of strength eps centred at the origin in a freestream
    of Mach `mach` along (1,1), rho = p = 1 (the vortex of ele::setInitialCondition,
    src/ele.cpp:708-733, with the strength and freestream as parameters)."""
    ui = mach * np.sqrt(gamma) / np.sqrt(2.0)
    x, y = pos[..., 0], pos[..., 1]
    f = 1.0 - (x * x + y * y)
    rho = (1.0 - eps * eps * (gamma - 1.0) / (8.0 * gamma * np.pi ** 2) * np.exp(f)) ** (1.0 / (gamma - 1.0))
    u = ui - eps * y / (2 * np.pi) * np.exp(f / 2)
    v = ui + eps * x / (2 * np.pi) * np.exp(f / 2)
    p = rho ** gamma
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)], axis=-1)


def run_ensemble(stream, nsteps=500, warmup=3, alone_steps=20, adj_steps=100):
    """Batched ensemble: the 256 cases grouped by order, each group one handle
    in ensemble mode (per-case CFL dt), the four handles advanced by one graph
    launch per step; against the same cases run one by one.  Then the adjoint
    of each case's final entropy error (FP64, per-case dt frozen at the first
    step's CFL value), per order group."""
    import torch

    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Ensemble, Solver, box2d, concat_meshes

    cases = ensemble_cases()
    kw = dict(riemannType=1, timeType=4, CFL=0.5, gamma=1.4)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
        return a.elapsed_time(b)

    meshes = {c["seed"]: box2d(c["side"], c["side"], -10, 10, -10, 10, perturb=0.1, seed=c["seed"]) for c in cases}
    groups = {}
    for c in cases:
        groups.setdefault(c["P"], []).append(c)
    solvers, tiles, total_dof, first_dt = [], {}, 0, {}
    for P in sorted(groups):
        cs = groups[P]
        union, grp = concat_meshes([meshes[c["seed"]] for c in cs])
        s = Solver(union, order=P, dtType=1, precision=FRG_MIXED, **kw)
        s.set_groups(grp, len(cs))
        pos = s.get("pos_spts")
        U = np.empty((s.nSpts, s.nEles, 4))
        for k, c in enumerate(cs):
            U[:, grp == k] = vortex_state(pos[:, grp == k], c["eps"], c["mach"])
        s.set("U_spts", U)
        s.set_stream(stream.cuda_stream)
        with torch.cuda.stream(stream):
            tiles[P] = int(s.autotune(5)[0])
        solvers.append((P, s, union, grp, U))
        total_dof += s.nEles * s.nSpts * s.nFields
    ens = Ensemble([s for _, s, _, _, _ in solvers])
    ens.set_stream(stream.cuda_stream)
    ens.update(warmup)
    for P, s, _, _, _ in solvers:
        first_dt[P] = s.group_times()[1]
    ms = timed(lambda: ens.update(nsteps))
    launches = sum(s.launch_count() for _, s, _, _, _ in solvers)
    ens.close()
    ens_rate = total_dof * nsteps / (ms * 1e-3)

    # the same cases one by one (own handle each, graph-replayed steps)
    alone_ms, alone_dof = 0.0, 0
    for c in cases:
        s = Solver(meshes[c["seed"]], order=c["P"], dtType=1, precision=FRG_MIXED, **kw)
        s.set("U_spts", vortex_state(s.get("pos_spts"), c["eps"], c["mach"]))
        s.set_stream(stream.cuda_stream)
        with torch.cuda.stream(stream):
            s.update(warmup)
        alone_ms += timed(lambda: s.update(alone_steps))
        alone_dof += s.nEles * s.nSpts * s.nFields
        s.set_stream(None)
        s.close()
    alone_rate = alone_dof * alone_steps / (alone_ms * 1e-3)
    for _, s, _, _, _ in solvers:
        s.set_stream(None)
        s.close()

    # adjoint of the per-case entropy error, FP64, per order group: with the
    # automatic memory strategy (every stage state kept when that fits in half
    # of the free memory) and with checkpoints every 25 steps (recomputation
    # overlapped with the reversal)
    fwd_ms, adj_ms, kept = 0.0, {"auto": 0.0, "checkpoint_25": 0.0}, {}
    for P, _, union, grp, U in solvers:
        a = Solver(union, order=P, dtType=0, dt=1.0, precision=FRG_FP64, **kw)
        a.set_groups(grp, grp.max() + 1, first_dt[P])
        a.set("U_spts", U)
        a.set_stream(stream.cuda_stream)
        with torch.cuda.stream(stream):
            a.update(1)
        a.set("U_spts", U)
        fwd_ms += timed(lambda: a.update(adj_steps))
        for mode, every in (("checkpoint_25", 25), ("auto", -1)):
            # one untimed forward + reverse sweep first: the segment graphs and
            # the stage slots are made on first use (set-up, like the forward's
            # warm-up)
            for timed_run in (False, True):
                a.set("U_spts", U)
                with torch.cuda.stream(stream):
                    a.adjoint_forward(adj_steps, every)
                    a.objective("entropy")
                if timed_run:
                    adj_ms[mode] += timed(lambda: a.adjoint_backward())
                else:
                    with torch.cuda.stream(stream):
                        a.adjoint_backward()
            if mode == "auto":
                kept[str(P)] = a.adjoint_mode()
        a.set_stream(None)
        a.close()
    return {"workload": "256 isentropic-vortex cases, side {16..96}, P {2..5}, strength U[1,5], Mach U[0.1,0.6], "
                        "Roe, RK4, per-case CFL 0.5, mixed precision",
            "cases": len(cases), "cases_per_order": {str(P): len(groups[P]) for P in sorted(groups)},
            "total_dof": total_dof, "steps": nsteps, "tile_variant_per_order": {str(k): v for k, v in tiles.items()},
            "ensemble_value": ens_rate, "ensemble_ms_per_step": ms / nsteps, "unit": "DOF-updates/s",
            "one_by_one_value": alone_rate, "one_by_one_steps_per_case": alone_steps,
            "ensemble_over_one_by_one": ens_rate / alone_rate,
            "adjoint_fp64": {"steps": adj_steps, "forward_ms_per_step": fwd_ms / adj_steps,
                             "adjoint_ms_per_step": adj_ms["auto"] / adj_steps,
                             "adjoint_over_forward": adj_ms["auto"] / fwd_ms,
                             "checkpoint_every_per_order": kept,
                             "memory": "auto: every stage state kept when it fits in half of the free device memory "
                                       "(0 = all kept), else checkpoints every 25 steps",
                             "checkpoint_every_25": {"adjoint_ms_per_step": adj_ms["checkpoint_25"] / adj_steps,
                                                     "adjoint_over_forward": adj_ms["checkpoint_25"] / fwd_ms},
                             "objective": "per-case entropy error integral at the final time"}}


TGV_N, TGV_P, TGV_MA = 32, 3, 0.1
TGV_WORKLOAD = "ns3d_taylor_green_periodic_32x32x32_hex_P3_re1600_ma0.1_rusanov_ldg_rk44_dt5e-4"


def tgv_mesh():
    from fr_learn_b200 import box3d

    return box3d(TGV_N, TGV_N, TGV_N, (0.0, 0.0, 0.0), (2 * np.pi,) * 3)


def tgv_params(**kw):
    """Taylor-Green vortex: Re 1600 (rho0 = V0 = L = 1, mu = 1/1600, fixVis),
    Pr 0.71, Rusanov inviscid flux, LDG viscous flux with penFact 0 and
    tau 1 (the reference's defaults, src/input.cpp:290-291), RK4, dt 5e-4.
    At Ma 0.1 the sound speed is 10 V0 and the CFL-1 step of this mesh
    (ele::calcDt with getCFLLimit(3)) is 9.3e-4: dt 1e-3 diverges within a
    few dozen steps in the CPU restatement of the reference as well as here,
    so the workload runs at dt 5e-4 (CFL ~0.54)."""
    d = dict(order=TGV_P, equation=1, viscous=1, riemannType=0, timeType=4, dtType=0, dt=5e-4, gamma=1.4,
             mu_inf=1.0 / 1600.0, prandtl=0.71, fixVis=1, penFact=0.0, tau=1.0)
    d.update(kw)
    return d


def kinetic_energy(U, detJ, P, nDims=3):
    """Volume-averaged kinetic energy (1/|V|) * integral of rho |u|^2 / 2 by
    the solution points' Gauss quadrature (tensor-product weights times
    detJ); U is [spt][ele][field], detJ [spt][ele]."""
    w1 = np.polynomial.legendre.leggauss(P + 1)[1]
    w = w1
    for _ in range(nDims - 1):
        w = np.multiply.outer(w1, w).reshape(-1)  # spt index i fastest: w[i] * w[j] * w[k]
    wd = w[:, None] * detJ
    rho = U[..., 0]
    ke = 0.5 * (U[..., 1] ** 2 + U[..., 2] ** 2 + U[..., 3] ** 2) / rho
    return float(np.sum(wd * ke) / np.sum(wd))


def run_tgv(stream, flush, steps=50, warmup=3, hist_steps=400, hist_every=25):
    """3D compressible Navier-Stokes Taylor-Green vortex, 32^3 periodic
    linear hexes, P = 3 (64 solution points per element, 10,485,760 DOF):
    DOF-updates/s of the mixed and FP64 paths (CUDA events per step, L2
    flushed before each), per-stage launch times against the byte model, and
    the kinetic-energy history of both paths over `hist_steps` steps (the
    dissipation rate -dE_k/dt by central differences of the samples)."""
    import torch

    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver

    mesh = tgv_mesh()
    out = {"workload": TGV_WORKLOAD}
    hist = {}
    final = {}
    for name, prec in (("mixed", FRG_MIXED), ("fp64", FRG_FP64)):
        s = Solver(mesh, precision=prec, **tgv_params())
        s.set_stream(stream.cuda_stream)
        s.setInitialCondition(10, TGV_MA)
        detJ = s.get("detJac_spts")
        dof = s.nEles * s.nSpts * s.nFields
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                flush.fill_(1)
                s.update(1)
            stream.synchronize()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            l0 = s.launch_count()
            for k in range(steps):
                flush.fill_(k & 0xFF)
                ev[k][0].record(stream)
                s.update(1)
                ev[k][1].record(stream)
            stream.synchronize()
            ms = sum(a.elapsed_time(b) for a, b in ev) / steps
            launches = (s.launch_count() - l0) / steps
            st = s.time_stages(max(3, min(10, steps)), flush.data_ptr(), flush.numel()).tolist()
        # kinetic-energy history from the initial condition
        s.setInitialCondition(10, TGV_MA)
        t_start = s.time
        ke, tt = [kinetic_energy(s.get("U_spts"), detJ, TGV_P)], [0.0]
        with torch.cuda.stream(stream):
            for _ in range(hist_steps // hist_every):
                s.update(hist_every)
                stream.synchronize()
                ke.append(kinetic_energy(s.get("U_spts"), detJ, TGV_P))
                tt.append(s.time - t_start)
        hist[name] = (np.array(tt), np.array(ke))
        final[name] = s.get("U_spts")
        b = bytes_per_dof_update(3, TGV_P, 5, 4 if prec == FRG_MIXED else 8, 4 if prec == FRG_MIXED else 8,
                                 viscous=True) / 4 * dof
        st_mean = float(np.mean(st[1:]))
        out[name] = {"value": dof / (ms * 1e-3), "ms_per_step": ms, "unit": "DOF-updates/s", "dof": dof,
                     "launches_per_step": launches, "stage_ms": st_mean, "bytes_per_stage": b,
                     "achieved_gbs": b / (st_mean * 1e-3) / 1e9,
                     "hbm_frac": b / (st_mean * 1e-3) / 1e9 / peaks()[0]}
        s.set_stream(None)
        s.close()
    (tm, km), (td, kd) = hist["mixed"], hist["fp64"]
    Um, Ud = final["mixed"], final["fp64"]
    out["state_error_mixed_vs_fp64"] = {"steps": hist_steps, "rel_l2": float(np.linalg.norm(Um - Ud) / np.linalg.norm(Ud)),
                                        "rel_linf": float(np.abs(Um - Ud).max() / np.abs(Ud).max())}
    eps_m = -np.gradient(km, tm)
    eps_d = -np.gradient(kd, td)
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["kinetic_energy"] = {
        "t": td.tolist(), "fp64": kd.tolist(), "mixed": km.tolist(),
        "max_rel_diff": float(np.max(np.abs(km - kd) / kd)),
        "dissipation_rate_fp64": eps_d.tolist(),
        "dissipation_rate_max_rel_diff": float(np.max(np.abs(eps_m - eps_d)) / np.max(np.abs(eps_d))),
    }
    return out


def run_tgv_oracle(stream, full_steps=2, small_n=8, small_steps=100, every=20):
    """Kinetic energy of the Taylor-Green workload against the FP64 oracle
    (the CPU restatement of the reference, on all host cores): (a) the full
    32^3 mesh for `full_steps` steps, (b) the same physics on a small_n^3
    mesh for `small_steps` steps, sampled every `every` steps, with the
    dissipation rate -dE_k/dt; both GPU paths (mixed, FP64) beside the
    oracle.  Bounded so the whole run stays within a few minutes."""
    import torch

    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver, box3d

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api

    oracle_api.lib().orc_set_threads(max(1, min(os.cpu_count() or 1, 64)))
    out = {}
    for label, mesh, nsteps, samp in (("full_32x32x32", tgv_mesh(), full_steps, 1),
                                      (f"small_{small_n}x{small_n}x{small_n}",
                                       box3d(small_n, small_n, small_n, (0.0, 0.0, 0.0), (2 * np.pi,) * 3),
                                       small_steps, every)):
        t0 = time.perf_counter()
        o = oracle_api.Oracle(oracle_api.params(nDims=3, **tgv_params()), mesh)
        o.set_ic(10, TGV_MA)
        detJ = o.get("detJac_spts").reshape(-1, mesh.nEles)
        ke = {"oracle_fp64": [kinetic_energy(o.U(), detJ, TGV_P)]}
        tt = [0.0]
        for _ in range(nsteps // samp):
            o.update(samp)
            ke["oracle_fp64"].append(kinetic_energy(o.U(), detJ, TGV_P))
            tt.append(o.time)
        o_s = time.perf_counter() - t0
        o.close()
        for name, prec in (("gpu_mixed", FRG_MIXED), ("gpu_fp64", FRG_FP64)):
            s = Solver(mesh, precision=prec, **tgv_params())
            s.set_stream(stream.cuda_stream)
            s.setInitialCondition(10, TGV_MA)
            ke[name] = [kinetic_energy(s.get("U_spts"), detJ, TGV_P)]
            with torch.cuda.stream(stream):
                for _ in range(nsteps // samp):
                    s.update(samp)
                    stream.synchronize()
                    ke[name].append(kinetic_energy(s.get("U_spts"), detJ, TGV_P))
            s.set_stream(None)
            s.close()
        t = np.array(tt)
        ref = np.array(ke["oracle_fp64"])
        eps_ref = -np.gradient(ref, t)
        r = {"steps": nsteps, "every": samp, "t": tt, "kinetic_energy": ke, "oracle_seconds": o_s}
        for name in ("gpu_mixed", "gpu_fp64"):
            k = np.array(ke[name])
            r[f"{name}_max_rel_diff"] = float(np.max(np.abs(k - ref) / ref))
            if len(t) > 2:
                r[f"{name}_dissipation_rate_max_rel_diff"] = float(np.max(np.abs(-np.gradient(k, t) - eps_ref))
                                                                   / np.max(np.abs(eps_ref)))
        out[label] = r
    return out


def time_device_metrics(s, mesh, nx, reps=4):
    """frg_update_geometry on the production-size mesh (moved nodes in, every
    metric recomputed on the device, positions and detJ copied back), wall
    time per call, next to the host set-up of the same metrics plus the face
    connectivity (build_geometry, one call of frg_inspect_geometry)."""
    import ctypes as C
    import time

    from fr_learn_b200 import box2d
    from fr_learn_b200.solver import MeshC, Params, default_params, lib

    moved = box2d(nx, nx, -10.0, 10.0, -10.0, 10.0, perturb=0.1, seed=1).xv
    s.update_geometry(moved)  # first call allocates the node and table buffers
    t0 = time.perf_counter()
    for k in range(reps):
        s.update_geometry(mesh.xv if k % 2 else moved)
    dev_ms = (time.perf_counter() - t0) / reps * 1e3
    L = lib()
    L.frg_inspect_geometry.argtypes = [C.POINTER(Params), C.POINTER(MeshC), C.c_int, C.c_void_p, C.POINTER(C.c_long)]
    L.frg_inspect_geometry.restype = C.c_int
    p = Params(**default_params(nDims=2, **c2_params()))
    xv = np.ascontiguousarray(mesh.xv, np.float64)
    c2v = np.ascontiguousarray(mesh.c2v, np.int32)
    bc = np.ascontiguousarray(mesh.bc, np.int32)
    m = MeshC(mesh.nEles, mesh.nNodes, xv.ctypes.data, c2v.ctypes.data, bc.ctypes.data)
    n = C.c_long()
    t0 = time.perf_counter()
    rc = L.frg_inspect_geometry(C.byref(p), C.byref(m), 2, None, C.byref(n))
    host_ms = (time.perf_counter() - t0) * 1e3
    return {"nEles": mesh.nEles, "device_update_ms": dev_ms, "host_setup_ms": host_ms if rc == 0 else None,
            "note": "device: H2D of the nodes, Jacobian check pass, metric and face kernels, positions and "
                    "detJ back to the host; host: metrics plus face connectivity, one thread"}


def run_scale(stream, flush, nx=512, steps=30):
    """The headline workload's physics at production size: the same vortex
    on 512 x 512 perturbed quads (262,144 elements, P = 4, 26.2 M DOF; a
    mixed step moves ~5.6 GB, far beyond L2), mixed and FP64, each with its
    autotuned tile variant; DOF-updates/s and the per-stage roofline
    fraction."""
    import torch

    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver, box2d

    mesh = box2d(nx, nx, -10.0, 10.0, -10.0, 10.0, perturb=0.1, seed=0)
    out = {"workload": f"euler2d_isentropic_vortex_periodic_{nx}x{nx}_P4_roe_rk44_cfl0.5", "nEles": nx * nx}
    for name, prec, sz in (("mixed", FRG_MIXED, 4), ("fp64", FRG_FP64, 8)):
        s = Solver(mesh, precision=prec, **c2_params())
        s.set_stream(stream.cuda_stream)
        s.setInitialCondition(1)
        with torch.cuda.stream(stream):
            var = int(s.autotune(5)[0])
            s.update(3)
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            for k in range(steps):
                flush.fill_(k & 0xFF)
                ev[k][0].record(stream)
                s.update(1)
                ev[k][1].record(stream)
            stream.synchronize()
            st = s.time_stages(10, flush.data_ptr(), flush.numel()).tolist()
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        dof = s.nEles * s.nSpts * s.nFields
        b = bytes_per_dof_update(2, ORDER, 4, sz, sz) / 4 * dof
        st_mean = float(np.mean(st[1:]))
        out["dof"] = dof
        out[name] = {"tile_variant": var, "value": dof / (ms * 1e-3), "ms_per_step": ms, "unit": "DOF-updates/s",
                     "stage_ms": st_mean, "bytes_per_stage": b, "achieved_gbs": b / (st_mean * 1e-3) / 1e9,
                     "hbm_frac": b / (st_mean * 1e-3) / 1e9 / peaks()[0]}
        if name == "mixed":
            out["device_metrics"] = time_device_metrics(s, mesh, nx)
        s.set_stream(None)
        s.close()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


C1_WORKLOAD = "advection2d_gaussian_periodic_32x32_P3_upwind_rk44_dt1e-3_1000steps"


def c1_mesh():
    from fr_learn_b200 import box2d

    return box2d(32, 32, -5.0, 5.0, -5.0, 5.0)


def c1_params(**kw):
    """Scalar advection at (1,1), Lax-Friedrichs flux with lambda 1 (upwind),
    DG correction, RK4, fixed dt 1e-3 (FP64)."""
    d = dict(order=3, equation=0, advectVx=1.0, advectVy=1.0, lambda_=1.0, timeType=4, dtType=0, dt=1e-3)
    d.update(kw)
    return d


def run_advection_c1(stream, nsteps=1000):
    """2D scalar advection of u0 = exp(-(x^2+y^2)) on the periodic square
    [-5,5]^2, 32 x 32 linear quads, P = 3, FP64, 1000 RK4 steps of 1e-3:
    DOF-updates/s over the run (CUDA events), and the relative L2 error at
    t = 1 against the exact solution (the bump translated by (1,1))."""
    import torch

    from fr_learn_b200 import FRG_FP64, Solver

    s = Solver(c1_mesh(), precision=FRG_FP64, **c1_params())
    s.set_stream(stream.cuda_stream)
    s.setInitialCondition(0)
    with torch.cuda.stream(stream):
        s.update(3)  # warm-up (graphs, kernels)
        s.setInitialCondition(0)
        s.setIter(0, 0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = s.time
        a.record(stream)
        s.update(nsteps)
        b.record(stream)
        b.synchronize()
    ms = a.elapsed_time(b)
    t = s.time - t0
    pos, U = s.get("pos_spts"), s.get("U_spts")[..., 0]
    x = np.mod(pos[..., 0] - t + 5.0, 10.0) - 5.0
    y = np.mod(pos[..., 1] - t + 5.0, 10.0) - 5.0
    ex = np.exp(-(x * x + y * y))
    dof = s.nEles * s.nSpts * s.nFields
    s.set_stream(None)
    s.close()
    return {"workload": C1_WORKLOAD, "dof": dof, "steps": nsteps, "time": t, "ms_per_step": ms / nsteps,
            "value_fp64": dof * nsteps / (ms * 1e-3), "unit": "DOF-updates/s",
            "rel_l2_vs_exact": float(np.linalg.norm(U - ex) / np.linalg.norm(ex)),
            "note": "16,384 DOF: launch-latency bound (4 stage launches per step from one graph)"}


def run_operator_gemm(stream, flush, reps=20):
    """The oper::apply* products as batched tensor-core GEMMs
    (frg_apply_operator: tcgen05 MMAs in 3xTF32, TMA-fed tiles) over the
    Taylor-Green mesh's arrays (32^3 hexes, P = 3, 5 fields, FP32): per
    operator the kernel time (CUDA events around the launch, L2 flushed
    before each), the HBM bytes it must move (X read, Y written), and the
    tensor throughput counting the three TF32 MMAs of each product."""
    import torch

    from fr_learn_b200 import FRG_MIXED, Solver

    s = Solver(tgv_mesh(), precision=FRG_MIXED, **tgv_params())
    s.set_stream(stream.cuda_stream)
    nV, nE, nS, nF = s.nFields, s.nEles, s.nSpts, s.nFpts
    ld = (nE + 31) // 32 * 32
    hbm = peaks()[0]
    out = {"workload": f"{nE} hexes x {nV} fields, P={TGV_P}, FP32 arrays [field][point][element]",
           "precision": "3xTF32 products, FP32 accumulation in TMEM", "ops": {}}
    for which, name, (M, K) in ((0, "spts_to_fpts", (nF, nS)), (1, "grad_spts_x", (nS, nS)),
                                (3, "correction", (nS, nF))):
        X = torch.randn((nV, K, ld), dtype=torch.float32, device=stream.device)
        Y = torch.empty((nV, M, ld), dtype=torch.float32, device=stream.device)
        with torch.cuda.stream(stream):
            for _ in range(3):
                s.apply_operator(which, 0, X.data_ptr(), Y.data_ptr(), ld)
            s.sync()
            ms = []
            for r in range(reps):
                flush.fill_(r & 0xFF)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                s.apply_operator(which, 0, X.data_ptr(), Y.data_ptr(), ld)
                b.record(stream)
                b.synchronize()
                ms.append(a.elapsed_time(b))
            s.sync()
        t = float(np.median(ms)) * 1e-3
        byt = 4.0 * nV * nE * (K + M)
        fl = 2.0 * M * K * nV * nE
        out["ops"][name] = {"M": M, "K": K, "ms": t * 1e3, "gbs": byt / t / 1e9, "hbm_frac": byt / t / 1e9 / hbm,
                            "useful_tflops": fl / t / 1e12, "tensor_tflops_3xtf32": 3 * fl / t / 1e12}
    # the operator products of ONE viscous RK stage as the reference applies
    # them (dense GEMMs at its dgemm sites, src/solver.cpp:401-412, :707-895),
    # here as tensor-core GEMMs back to back: E U; D_d U (3); correctU_d dUc
    # (3, beta 1); E dU_d (3); Efn_d F_d (3); D_d F_d (3, beta 1 after the
    # first); C (Fn - disFn) (beta 1) -- 17 launches, timed as one sequence
    # with L2 flushed before it.  The fused stage applies the same operators
    # by sum factorisation on data that stays in shared memory.
    seq = [(0, 0, nF, nS, 0.0)] + [(1, d, nS, nS, 0.0) for d in range(3)] + \
          [(4, d, nS, nF, 1.0) for d in range(3)] + [(0, 0, nF, nS, 0.0) for d in range(3)] + \
          [(2, d, nF, nS, 0.0) for d in range(3)] + [(1, d, nS, nS, 0.0 if d == 0 else 1.0) for d in range(3)] + \
          [(3, 0, nS, nF, 1.0)]
    bufs = {(M, K): (torch.randn((nV, K, ld), dtype=torch.float32, device=stream.device),
                     torch.zeros((nV, M, ld), dtype=torch.float32, device=stream.device))
            for (_, _, M, K, _) in seq}
    with torch.cuda.stream(stream):
        ms = []
        for r in range(5):
            flush.fill_(r & 0xFF)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for which, d, M, K, beta in seq:
                X, Y = bufs[(M, K)]
                s.apply_operator(which, d, X.data_ptr(), Y.data_ptr(), ld, beta)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        s.sync()
    out["viscous_stage_as_dense_gemms"] = {
        "launches": len(seq), "ms": float(np.median(ms[1:])),
        "note": "operator products alone (no fluxes, no Riemann solver, no RK update); compare "
                "taylor_green_3d.<mode>.stage_ms, the whole fused stage"}
    s.set_stream(None)
    s.close()
    return out


def cpu_baseline(steps=2, threads=1):
    """The oracle (CPU restatement of the reference, which cannot run 2D
    meshes) on the same workload, timed on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api

    oracle_api.lib().orc_set_threads(threads)
    mesh = c2_mesh()
    p = oracle_api.params(nDims=2, **c2_params())
    o = oracle_api.Oracle(p, mesh)
    o.set_ic(1)
    o.update(1)  # first iteration also recomputes the wave speeds
    t0 = time.perf_counter()
    o.update(steps)
    dt = time.perf_counter() - t0
    dof = o.nE * o.nS * o.nV
    return dof * steps / dt, dt


def profile_run(case, variant=None):
    """A few steps of one workload and nothing else, for profiler captures
    (`ncu ... python bench.py --profile CASE`): builds the handle, runs,
    synchronises and returns.  Cases: c2_mixed / c2_fp64 (the 2D vortex
    workload, 4 steps, L2 flushed before each as in the timed region;
    `variant` picks the stage kernel's tile shape),
    tgv_mixed / tgv_fp64 (3D Taylor-Green, 32^3 hexes, P = 3, 2 steps),
    opgemm (the tensor-core operator GEMMs over the Taylor-Green arrays:
    spts->fpts, grad_x, correction, 2 calls each)."""
    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver

    prec = FRG_FP64 if case.endswith("fp64") else FRG_MIXED
    if case.startswith("c2"):
        import torch

        # as in the timed region: L2 flushed (a 512 MiB write) before every step
        flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
        s = Solver(c2_mesh(), precision=prec, **c2_params())
        s.set_stream(torch.cuda.current_stream().cuda_stream)
        s.setInitialCondition(1)
        if variant is not None:
            s.set_tile_variant(int(variant))
        for k in range(4):
            flush.fill_(k)
            s.update(1)
        s.sync()
        print(case, "time", s.time)
        s.set_stream(None)
    elif case.startswith("tgv"):
        s = Solver(tgv_mesh(), precision=prec, **tgv_params())
        s.setInitialCondition(10, TGV_MA)
        s.update(2)
        s.sync()
        print(case, "time", s.time)
    elif case == "opgemm":
        import torch

        s = Solver(tgv_mesh(), precision=FRG_MIXED, **tgv_params())
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
        raise SystemExit(f"unknown profile case {case!r}")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile", nargs="+", metavar=("CASE", "VARIANT"),
                    help="run a few steps of one workload for a profiler capture, then exit")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--tile-variants", metavar="MIXED,FP64",
                    help="stage-kernel tile variants of the headline workload instead of autotuning them "
                         "(e.g. for a profiler launch list, whose serialisation changes the autotuner's pick)")
    args = ap.parse_args()
    if args.profile:
        return profile_run(args.profile[0], args.profile[1] if len(args.profile) > 1 else None)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    n = max(args.gpus, world)

    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = max(1, min(os.cpu_count() or 1, 64))
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_api

        oracle_api.lib().orc_set_threads(threads)
        mesh = c2_mesh()
        o = oracle_api.Oracle(oracle_api.params(nDims=2, **c2_params()), mesh)
        o.set_ic(1)
        dof = o.nE * o.nS * o.nV
        # bounded sample: at most 3 warm-up steps and ~60 s of timed steps
        for _ in range(min(args.warmup, 3)):
            o.update(1)
        t0 = time.perf_counter()
        done = 0
        while done < args.steps and (done == 0 or time.perf_counter() - t0 < 60.0):
            o.update(1)
            done += 1
        secs = time.perf_counter() - t0
        v = dof * done / secs
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": n, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * secs / done, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "nEles": o.nE, "order": ORDER, "dof": dof},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"{done} RK4 steps of the full workload (bounded to ~60 s) after "
                                           f"{min(args.warmup, 3)} warm-up steps"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference cannot run 2D meshes (src/geo.cpp:35-37); this arm times the oracle, "
                        "its CPU restatement, which reproduces the reference bit-for-bit on 3D cases"}
        print(json.dumps(line))
        return 0

    if world > 1:
        import torch

        torch.distributed.init_process_group("nccl", init_method="env://",
                                             timeout=__import__("datetime").timedelta(seconds=120))
    dof, res, stage_ms, clocks, errs, (e2e_ms, state_bytes, copy_ms) = run_gpu(args, rank, world, local_rank)
    if rank != 0:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
        return 0
    mixed, fp64 = res["mixed"], res["fp64"]
    tiles = res["tile_variant"]
    value = throughput(n, dof, mixed["ms_per_step"])
    value_fp64 = throughput(n, dof, fp64["ms_per_step"])
    peak, peak_kind = peaks()
    # dominant kernel: the fused RK stage kernel (mean over the 4 stages)
    st_mixed = float(np.mean(stage_ms["mixed"][1:]))
    st_fp64 = float(np.mean(stage_ms["fp64"][1:]))
    b_mixed = bytes_per_dof_update(2, ORDER, 4, 4, 4) / 4 * dof  # per stage launch
    b_fp64 = bytes_per_dof_update(2, ORDER, 4, 8, 8) / 4 * dof
    ach = b_mixed / (st_mixed * 1e-3) / 1e9
    ach64 = b_fp64 / (st_fp64 * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "stage_tma_split_kernel_euler2d_vortex_128x128_P4_traffic.json.txt")
    if os.path.exists(tp):
        try:
            with open(tp) as f:
                traffic = json.load(f).get("mixed_dram_bytes_per_launch")
        except (OSError, ValueError):
            traffic = None
    cpu_v, cpu_s = cpu_baseline(steps=2, threads=1)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mixed["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 operators/fluxes + f64 Riemann pressure & RK accumulation (mixed)",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "nEles": NX * NX, "order": ORDER, "dof": dof, "parallelism":
                   f"replicas x{n}" if n > 1 else "single GPU", "l2": "flushed (512 MiB write) before every step",
                   "tile_variant": tiles},
        "fp64": {"value": value_fp64, "ms_per_step": fp64["ms_per_step"], "unit": UNIT},
        "mixed_over_fp64": value / value_fp64,
        "error_vs_fp64": {"rel_l2": errs[0], "rel_linf": errs[1], "steps": args.warmup + args.steps,
                          "time": errs[3]},
        "fp64_density_rel_l2_vs_exact_vortex": errs[2],
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "traffic_source": "static: dram__bytes_read.sum + dram__bytes_write.sum per stage launch, the "
                                       "mean over the four RK stages of one step, each replayed from a clean L2, from "
                                       "the committed ncu capture of the split kernel (profiles/); not measured in "
                                       "this run",
                     "kernel": ("fr_stage_tma_split_kernel" if tiles["mixed"] >= 10 else "fr_stage_tma_pipe_kernel"
                                if tiles["mixed"] >= 6 else "fr_stage_tma_kernel")
                               + f" (mixed, tile variant {tiles['mixed']})", "launch_ms": st_mixed,
                     "bytes_per_launch": b_mixed,
                     "fp64": {"achieved": ach64, "frac": ach64 / peak, "launch_ms": st_fp64,
                              "bytes_per_launch": b_fp64},
                     "pre_stage_ms": stage_ms["mixed"][0],
                     "pre_stage_note": "event interval before the first stage: the dt kernel when the previous "
                                       "step did not compute dt, else empty (event overhead)"},
        "cpu_baseline": {"value": cpu_v, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": f"2 RK4 steps of the full 128x128 P4 workload ({cpu_s:.1f} s), oracle "
                                   "(CPU restatement; the reference cannot run 2D meshes)"},
        "l2_resident": {"value": throughput(n, dof, mixed["l2_resident_ms_per_step"]),
                        "ms_per_step": mixed["l2_resident_ms_per_step"],
                        "hbm_frac_per_stage": b_mixed / (mixed["l2_resident_ms_per_step"] / 4 * 1e-3) / 1e9 / peak,
                        "fp64_value": throughput(n, dof, fp64["l2_resident_ms_per_step"]),
                        "fp64_ms_per_step": fp64["l2_resident_ms_per_step"],
                        "how": "update(n) back to back with no L2 flush between steps (the working set stays in "
                               "L2, as in a long run); not the headline, which flushes before every step"},
        "e2e": {"value": throughput(n, dof, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes,
                "how": "frg_update_host per step: pinned host state [spt][ele][field] -> device, one RK4 step, "
                       "state -> host",
                "host_link_bound": {"copy_ms": copy_ms, "gbs": 2 * state_bytes / (copy_ms * 1e-3) / 1e9,
                                    "step_ms_at_bound": copy_ms + mixed["ms_per_step"],
                                    "frac": (copy_ms + mixed["ms_per_step"]) / e2e_ms,
                                    "how": "one pinned H2D and one D2H copy of the state (torch copies, same "
                                           "stream), plus the device-timed step; frac = that sum / the e2e step"}},
        "adjoint": res["adjoint"],
        "ensemble": res["ensemble"],
        "taylor_green_3d": res["tgv"],
        "advection_2d": res["c1"],
        "euler2d_at_scale": res["scale"],
        "operator_gemm_tensor_cores": res["opgemm"],
        "gpu_launches": mixed["launches"],
        "clocks": clocks,
    }
    print(json.dumps(line))
    if world > 1:
        import torch

        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
