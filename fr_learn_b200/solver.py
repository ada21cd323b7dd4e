"""Python mirror of FlurryPP's solver entry points over the libfrgpu C ABI.

Method names follow the reference's `solver` (include/solver.hpp:137-153):
``calcResidual``, ``update``, ``timeStepA``, ``timeStepB``, ``copyUspts_U0``,
``copyU0_Uspts``, ``calcDt``, plus ``getNormResidual`` (writeResidual's sum of
ele::getNormResidual) and the ``input`` parameter names.  Arrays cross the
boundary in the reference's layouts ([point][element][field]).

There is no CPU fallback: importing works without a GPU, but creating a
Solver raises if libfrgpu.so is missing or no CUDA device is usable.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .mesh import Mesh

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfrgpu.so")

FRG_FP64, FRG_MIXED = 0, 1
ARRAYS = {"U_spts": 0, "U0": 1, "divF_spts": 2, "U_fpts": 3, "pos_spts": 4, "waveSp": 5, "detJac_spts": 6,
          "ele_dt": 7}
STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NAN", 4: "ERR_NEG_JAC", 5: "ERR_DT", 6: "ERR_TIMEOUT",
          7: "ERR_MESH"}


class FrgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("nDims", C.c_int), ("order", C.c_int), ("equation", C.c_int), ("viscous", C.c_int),
        ("riemannType", C.c_int), ("vcjhScheme", C.c_int), ("timeType", C.c_int), ("dtType", C.c_int),
        ("dt", C.c_double), ("CFL", C.c_double), ("gamma", C.c_double),
        ("advectVx", C.c_double), ("advectVy", C.c_double), ("advectVz", C.c_double),
        ("lambda_", C.c_double), ("diffD", C.c_double),
        ("rhoBound", C.c_double), ("uBound", C.c_double), ("vBound", C.c_double),
        ("wBound", C.c_double), ("pBound", C.c_double),
        ("mu_inf", C.c_double), ("prandtl", C.c_double), ("c_sth", C.c_double), ("rt_inf", C.c_double),
        ("fixVis", C.c_int), ("penFact", C.c_double), ("tau", C.c_double),
        ("TWall", C.c_double), ("RGas", C.c_double), ("uWall", C.c_double), ("vWall", C.c_double),
        ("wWall", C.c_double), ("precision", C.c_int),
    ]


class MeshC(C.Structure):
    _fields_ = [("nEles", C.c_int), ("nNodes", C.c_int), ("xv", C.c_void_p), ("c2v", C.c_void_p),
                ("bc", C.c_void_p)]


def default_params(**kw) -> dict:
    """Defaults of input::readInputFile (src/input.cpp:214-475)."""
    d = dict(nDims=2, order=3, equation=1, viscous=0, riemannType=0, vcjhScheme=0, timeType=4, dtType=0,
             dt=1e-3, CFL=0.5, gamma=1.4, advectVx=1.0, advectVy=1.0, advectVz=0.0, lambda_=1.0, diffD=1.0,
             rhoBound=1.0, uBound=0.2, vBound=0.0, wBound=0.0, pBound=0.7142857143,
             mu_inf=1.0 / 1600.0, prandtl=0.72, c_sth=0.0, rt_inf=1.0, fixVis=1, penFact=0.0, tau=1.0,
             TWall=1.0, RGas=1.0, uWall=0.0, vWall=0.0, wWall=0.0, precision=FRG_FP64)
    if "lambda" in kw:
        kw["lambda_"] = kw.pop("lambda")
    d.update(kw)
    return d


_lib = None


def lib():
    """Loads libfrgpu.so (building it if this is a source checkout without it)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _b
        _b.build()
    L = C.CDLL(LIB_PATH)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    sig = {
        "frg_last_error": ([], C.c_char_p), "frg_version": ([], C.c_char_p),
        "frg_create": ([C.POINTER(Params), C.POINTER(MeshC), C.POINTER(vp)], i),
        "frg_destroy": ([vp], i),
        "frg_info": ([vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i)], i),
        "frg_update_geometry": ([vp, vp], i),
        "frg_write_paraview": ([vp, C.c_char_p], i), "frg_read_restart": ([vp, C.c_char_p, i], i),
        "frg_write_paraview_host": ([C.POINTER(Params), C.POINTER(MeshC), vp, d, i, C.c_char_p], i),
        "frg_read_restart_host": ([C.POINTER(Params), i, C.c_char_p, i, vp, C.POINTER(d)], i),
        "frg_get_operator": ([vp, i, i, vp], i),
        "frg_apply_operator": ([vp, i, i, vp, vp, i, C.c_float], i),
        "frg_upload": ([vp, i, vp], i), "frg_download": ([vp, i, i, vp], i),
        "frg_set_initial_condition": ([vp, i, d], i),
        "frg_calc_residual": ([vp, i], i), "frg_time_step_a": ([vp, i, d], i), "frg_time_step_b": ([vp, i], i),
        "frg_copy_u_to_u0": ([vp], i), "frg_copy_u0_to_u": ([vp], i),
        "frg_calc_dt": ([vp, C.POINTER(d)], i), "frg_update": ([vp, i], i), "frg_update_host": ([vp, vp, i], i),
        "frg_residual_norm": ([vp, i, vp], i), "frg_set_monitor": ([vp, i], i),
        "frg_get_time": ([vp, C.POINTER(d), C.POINTER(d), C.POINTER(i)], i),
        "frg_set_iter": ([vp, i, i], i), "frg_sync": ([vp], i),
        "frg_launch_count": ([vp, C.POINTER(C.c_longlong)], i),
        "frg_set_stream": ([vp, vp], i),
        "frg_calc_residual_noalloc": ([vp, vp, vp, vp], i),
        "frg_time_stages": ([vp, i, vp, C.c_ulonglong, vp], i),
        "frg_autotune": ([vp, i, C.POINTER(C.c_int), vp], i),
        "frg_set_tile_variant": ([vp, i], i),
        "frg_tile_variant_count": ([vp, C.POINTER(i)], i),
        "frg_objective": ([vp, i, C.POINTER(d), vp], i),
        "frg_set_groups": ([vp, vp, i, vp], i),
        "frg_ensemble_create": ([vp, i, C.POINTER(vp)], i),
        "frg_ensemble_set_stream": ([vp, vp], i),
        "frg_ensemble_update": ([vp, i], i),
        "frg_ensemble_destroy": ([vp], i),
        "frg_get_group_times": ([vp, vp, vp], i),
        "frg_residual_vjp": ([vp, vp, vp, vp, C.POINTER(d)], i),
        "frg_adjoint_forward": ([vp, i, i], i),
        "frg_adjoint_mode": ([vp, C.POINTER(i)], i),
        "frg_adjoint_backward": ([vp, vp, vp, vp, C.POINTER(d)], i),
        "frg_read_gmsh": ([C.c_char_p, C.c_char_p, C.POINTER(i), C.POINTER(i), C.POINTER(i), vp, vp, vp], i),
        "frg_wall_force": ([vp, vp], i),
        "frg_set_operators": ([vp, i, vp, vp, vp, vp], i),
        "frg_mass_flux": ([vp, i, vp], i),
        "frg_integrate_error": ([vp, i, d, i, i, vp, vp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(code):
    if code != 0:
        raise FrgError(code, lib().frg_last_error().decode())


class Solver:
    """One FR solver on the current CUDA device (a drop-in for `solver`)."""

    def __init__(self, mesh: Mesh, **params):
        self.params = default_params(nDims=mesh.nDims, **params)
        self.mesh = mesh
        L = lib()
        p = Params(**self.params)
        xv = np.ascontiguousarray(mesh.xv, np.float64)
        c2v = np.ascontiguousarray(mesh.c2v, np.int32)
        bc = np.ascontiguousarray(mesh.bc, np.int32)
        m = MeshC(mesh.nEles, mesh.nNodes, xv.ctypes.data, c2v.ctypes.data, bc.ctypes.data)
        h = C.c_void_p()
        _check(L.frg_create(C.byref(p), C.byref(m), C.byref(h)))
        self.h = h
        nS, nF, nV, nE = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(L.frg_info(h, C.byref(nS), C.byref(nF), C.byref(nV), C.byref(nE)))
        self.nSpts, self.nFpts, self.nFields, self.nEles = nS.value, nF.value, nV.value, nE.value

    # -- lifetime
    def close(self):
        if getattr(self, "h", None):
            lib().frg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- data
    def _shape(self, name):
        nS, nF, nV, nE, d = self.nSpts, self.nFpts, self.nFields, self.nEles, self.params["nDims"]
        return {"U_spts": (nS, nE, nV), "U0": (nS, nE, nV), "divF_spts": (nS, nE, nV), "U_fpts": (nF, nE, nV),
                "pos_spts": (nS, nE, d), "waveSp": (nE, nF), "detJac_spts": (nS, nE), "ele_dt": (nE,)}[name]

    def get(self, name, stage=0):
        out = np.empty(self._shape(name), np.float64)
        _check(lib().frg_download(self.h, ARRAYS[name], stage, out.ctypes.data))
        return out

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, np.float64)
        assert a.shape == self._shape(name), (a.shape, self._shape(name))
        _check(lib().frg_upload(self.h, ARRAYS[name], a.ctypes.data))

    def operator(self, which, dim=0):
        nS, nF = self.nSpts, self.nFpts
        shape = {0: (nF, nS), 1: (nS, nS), 2: (nF, nS), 3: (nS, nF), 4: (nS, nF)}[which]
        out = np.empty(shape, np.float64)
        _check(lib().frg_get_operator(self.h, which, dim, out.ctypes.data))
        return out

    def set_operators(self, order, E, D, C, Efn=None):
        """oper::setupOperators's matrices for the device path (see
        include/frgpu.h frg_set_operators): E [nF][nS], D [nDims][nS][nS],
        C [nS][nF], Efn [nDims][nF][nS] or None."""
        arrs = [np.ascontiguousarray(a, np.float64) if a is not None else None for a in (E, D, C, Efn)]
        ptrs = [a.ctypes.data if a is not None else None for a in arrs]
        _check(lib().frg_set_operators(self.h, order, *ptrs))

    def apply_operator(self, which, dim, X_ptr, Y_ptr, ld, beta=0.0):
        """Y = Op X + beta Y on FP32 device arrays [nFields][points][ld] (the
        oper::apply* products as tensor-core GEMMs, see include/frgpu.h)."""
        _check(lib().frg_apply_operator(self.h, which, dim, X_ptr, Y_ptr, ld, beta))

    def update_geometry(self, xv):
        """Recomputes the metrics on the device for moved nodes xv
        [nEles][nNodes][nDims] of the same mesh (solver::updateTransforms)."""
        a = np.ascontiguousarray(xv, np.float64)
        assert a.shape == np.shape(self.mesh.xv), (a.shape, np.shape(self.mesh.xv))
        _check(lib().frg_update_geometry(self.h, a.ctypes.data))

    def write_paraview(self, dataFileName):
        """writeParaview: <dataFileName>_<iter:09d>.vtu of the current state."""
        _check(lib().frg_write_paraview(self.h, os.fsencode(dataFileName)))

    def read_restart(self, dataFileName, restartIter):
        """readRestartFile: state and time from <dataFileName>_<restartIter:09d>.vtu."""
        _check(lib().frg_read_restart(self.h, os.fsencode(dataFileName), restartIter))

    # -- the reference's entry points
    def setInitialCondition(self, icType=None, a0=0.0):
        _check(lib().frg_set_initial_condition(self.h, self.params.get("icType", 1) if icType is None else icType, a0))

    def calcResidual(self, step=0):
        _check(lib().frg_calc_residual(self.h, step))

    def calcResidual_noalloc(self, U_dev_ptr, divF_dev_ptr, stream_ptr=None):
        """Residual of a caller-owned device state into a caller-owned device
        array ([nFields][nSpts][nEles]), with no device allocation: for callers
        whose device memory is all pre-planned or owned by another manager.
        Traces go to the library's fixed 16 MiB scratch array (see
        include/frgpu.h); overlapping calls race on it."""
        _check(lib().frg_calc_residual_noalloc(self.h, U_dev_ptr, divF_dev_ptr, stream_ptr))

    def timeStepA(self, step, RKval):
        _check(lib().frg_time_step_a(self.h, step, RKval))

    def timeStepB(self, step):
        _check(lib().frg_time_step_b(self.h, step))

    def copyUspts_U0(self):
        _check(lib().frg_copy_u_to_u0(self.h))

    def copyU0_Uspts(self):
        _check(lib().frg_copy_u0_to_u(self.h))

    def calcDt(self):
        dt = C.c_double()
        _check(lib().frg_calc_dt(self.h, C.byref(dt)))
        return dt.value

    def update(self, nsteps=1):
        """nsteps iterations of the main loop body (iter++; solver::update())."""
        _check(lib().frg_update(self.h, nsteps))

    def update_host(self, U_host, nsteps=1):
        _check(lib().frg_update_host(self.h, U_host.ctypes.data, nsteps))

    def getNormResidual(self, normType=2):
        out = np.empty(self.nFields, np.float64)
        _check(lib().frg_residual_norm(self.h, normType, out.ctypes.data))
        return out

    def setMonitor(self, enable=True):
        _check(lib().frg_set_monitor(self.h, int(enable)))

    def setIter(self, it, initIter=0):
        _check(lib().frg_set_iter(self.h, it, initIter))

    @property
    def time(self):
        t, dt, it = C.c_double(), C.c_double(), C.c_int()
        _check(lib().frg_get_time(self.h, C.byref(t), C.byref(dt), C.byref(it)))
        return t.value

    @property
    def dt(self):
        t, dt, it = C.c_double(), C.c_double(), C.c_int()
        _check(lib().frg_get_time(self.h, C.byref(t), C.byref(dt), C.byref(it)))
        return dt.value

    @property
    def iter(self):
        t, dt, it = C.c_double(), C.c_double(), C.c_int()
        _check(lib().frg_get_time(self.h, C.byref(t), C.byref(dt), C.byref(it)))
        return it.value

    # -- output integrals (solver::computeWallForce / computeMassFlux /
    #    integrateError) of the current solution
    def computeWallForce(self):
        out = np.zeros(6)
        _check(lib().frg_wall_force(self.h, out.ctypes.data))
        return out

    def computeMassFlux(self, errorNorm=0):
        out = np.zeros(self.nFields)
        _check(lib().frg_mass_flux(self.h, errorNorm, out.ctypes.data))
        return out

    def integrateError(self, icType, errorNorm=1, quadOrder=10, box=(-5.0, 5.0, -5.0, 5.0), eps=5.0):
        out = np.zeros(self.nFields)
        b = np.ascontiguousarray(box, np.float64)
        _check(lib().frg_integrate_error(self.h, icType, eps, errorNorm, quadOrder, b.ctypes.data, out.ctypes.data))
        return out

    def sync(self):
        _check(lib().frg_sync(self.h))

    def launch_count(self):
        n = C.c_longlong()
        _check(lib().frg_launch_count(self.h, C.byref(n)))
        return n.value

    def set_stream(self, stream_ptr):
        """Run on a caller's cudaStream_t (an int handle, e.g. torch's
        ``stream.cuda_stream``); None restores the solver's own stream."""
        _check(lib().frg_set_stream(self.h, stream_ptr))

    def autotune(self, nsteps=5):
        """Pick the fastest tile shape of the fused stage kernel by timing
        `nsteps` steps of each candidate; the solution is left unchanged.
        Returns (chosen index, per-candidate ms per step)."""
        v = C.c_int()
        out = np.zeros(16)  # FRG_MAX_TILE_VARIANTS
        _check(lib().frg_autotune(self.h, nsteps, C.byref(v), out.ctypes.data))
        return v.value, out[:self.tile_variant_count()]

    def tile_variant_count(self):
        n = C.c_int()
        _check(lib().frg_tile_variant_count(self.h, C.byref(n)))
        return n.value

    # -- ensemble mode
    def set_groups(self, group_of_element, n_groups, fixed_dt=None):
        """Independent cases in one mesh: per-group CFL dt (or fixed_dt[g])
        and time; see frg_set_groups."""
        g = np.ascontiguousarray(group_of_element, np.int32)
        assert g.shape == (self.nEles,)
        self._groups = g
        fd = None
        if fixed_dt is not None:
            fd = np.ascontiguousarray(fixed_dt, np.float64)
            assert fd.shape == (n_groups,)
        self._fixed_dt = fd
        self.n_groups = n_groups
        _check(lib().frg_set_groups(self.h, g.ctypes.data, n_groups, None if fd is None else fd.ctypes.data))

    def group_times(self):
        """(time per group, dt of the last step per group)."""
        t = np.empty(self.n_groups)
        dt = np.empty(self.n_groups)
        _check(lib().frg_get_group_times(self.h, t.ctypes.data, dt.ctypes.data))
        return t, dt

    # -- discrete adjoint (FP64, inviscid, fixed dt)
    OBJECTIVES = {"entropy": 1, "wall_pressure": 2}

    def objective(self, kind):
        """(J, dJ/dU_spts) of the current state; kind "entropy" or "wall_pressure"."""
        J = C.c_double()
        g = np.empty(self._shape("U_spts"), np.float64)
        _check(lib().frg_objective(self.h, self.OBJECTIVES[kind], C.byref(J), g.ctypes.data))
        return J.value, g

    @staticmethod
    def _theta(theta_dir):
        if theta_dir is None:
            return None, None
        t = np.ascontiguousarray(theta_dir, np.float64)
        assert t.shape == (5,)
        return t, t.ctypes.data

    def residual_vjp(self, gbar, theta_dir=None):
        """(d divF/dU)^T gbar at the current state, and gbar . d divF/dtheta
        for the boundary-state direction theta_dir = d(rho, u, v, w, p)_B/dtheta."""
        g = np.ascontiguousarray(gbar, np.float64)
        assert g.shape == self._shape("U_spts")
        out = np.empty_like(g)
        tb = C.c_double()
        t, tp = self._theta(theta_dir)
        _check(lib().frg_residual_vjp(self.h, g.ctypes.data, tp, out.ctypes.data, C.byref(tb)))
        return out, tb.value

    def adjoint_forward(self, nsteps, checkpoint_every=25):
        """nsteps of update() keeping checkpoints for adjoint_backward()
        (checkpoint_every 0: every stage state kept; -1: every stage state
        kept if it fits in half of the free device memory, else 25)."""
        _check(lib().frg_adjoint_forward(self.h, nsteps, checkpoint_every))

    def adjoint_mode(self):
        """The last adjoint_forward run's checkpoint interval (0: all kept)."""
        k = C.c_int(0)
        _check(lib().frg_adjoint_mode(self.h, C.byref(k)))
        return k.value

    def adjoint_backward(self, lamN=None, theta_dir=None):
        """(dJ/dU_0, dJ/dtheta through the boundary state) for the last
        adjoint_forward run; lamN = dJ/dU_N, or None for the last objective()."""
        lam0 = np.empty(self._shape("U_spts"), np.float64)
        ptr = None
        if lamN is not None:
            lamN = np.ascontiguousarray(lamN, np.float64)
            assert lamN.shape == lam0.shape
            ptr = lamN.ctypes.data
        tb = C.c_double()
        t, tp = self._theta(theta_dir)
        _check(lib().frg_adjoint_backward(self.h, ptr, tp, lam0.ctypes.data, C.byref(tb)))
        return lam0, tb.value

    def set_tile_variant(self, v):
        """Select a tile shape of the fused stage kernel by index."""
        _check(lib().frg_set_tile_variant(self.h, v))

    def time_stages(self, nsteps, flush_ptr=None, flush_bytes=0):
        """Mean per-launch device time (ms) of [dt kernels, stage 0..nRK-1]."""
        nrk = {0: 1, 2: 2, 4: 4, 5: 4}[self.params["timeType"]]
        out = np.zeros(1 + nrk)
        _check(lib().frg_time_stages(self.h, nsteps, flush_ptr, flush_bytes, out.ctypes.data))
        return out


def inspect_geometry(mesh: Mesh, which: str, **params) -> np.ndarray:
    """Host-only: the metrics / face table frg_create would build (no GPU needed)."""
    items = {"pos_spts": 0, "JGinv_spts": 1, "detJac_spts": 2, "norm_fpts": 3, "dA_fpts": 4, "faces": 5}
    L = lib()
    L.frg_inspect_geometry.argtypes = [C.POINTER(Params), C.POINTER(MeshC), C.c_int, C.c_void_p,
                                       C.POINTER(C.c_long)]
    L.frg_inspect_geometry.restype = C.c_int
    p = Params(**default_params(nDims=mesh.nDims, **params))
    xv = np.ascontiguousarray(mesh.xv, np.float64)
    c2v = np.ascontiguousarray(mesh.c2v, np.int32)
    bc = np.ascontiguousarray(mesh.bc, np.int32)
    m = MeshC(mesh.nEles, mesh.nNodes, xv.ctypes.data, c2v.ctypes.data, bc.ctypes.data)
    n = C.c_long()
    _check(L.frg_inspect_geometry(C.byref(p), C.byref(m), items[which], None, C.byref(n)))
    out = np.empty(n.value, np.float64)
    _check(L.frg_inspect_geometry(C.byref(p), C.byref(m), items[which], out.ctypes.data, C.byref(n)))
    if which == "faces":
        return out.reshape(-1, 6).astype(np.int64)
    return out


def write_paraview_host(mesh: Mesh, U, time, iter, dataFileName, **params):
    """Host-only writeParaview of a state U [nSpts][nEles][nFields]."""
    params.setdefault("nDims", mesh.nDims)
    p = Params(**default_params(**params))
    xv = np.ascontiguousarray(mesh.xv, np.float64)
    m = MeshC(mesh.nEles, mesh.nNodes, xv.ctypes.data, None, None)
    u = np.ascontiguousarray(U, np.float64)
    _check(lib().frg_write_paraview_host(C.byref(p), C.byref(m), u.ctypes.data, float(time), int(iter),
                                         os.fsencode(dataFileName)))


def read_restart_host(nEles, dataFileName, restartIter, **params):
    """Host-only restart read: (U [nSpts][nEles][nFields], time)."""
    pd = default_params(**params)
    p = Params(**pd)
    n1 = pd["order"] + 1
    nS = n1 ** pd["nDims"]
    nV = 1 if pd["equation"] == 0 else pd["nDims"] + 2
    U = np.empty((nS, nEles, nV), np.float64)
    t = C.c_double(0.0)
    _check(lib().frg_read_restart_host(C.byref(p), int(nEles), os.fsencode(dataFileName), int(restartIter),
                                       U.ctypes.data, C.byref(t)))
    return U, t.value


def read_gmsh(fileName, meshBounds) -> Mesh:
    """geo::readGmsh: a Gmsh v2 ASCII file as a Mesh.  meshBounds maps the
    file's physical names to boundary conditions like the reference's
    ``mesh_bound`` lines: a dict {name: bc} or a "name bc; name bc" string,
    with one name mapped to "fluid" (the volume)."""
    if isinstance(meshBounds, dict):
        meshBounds = "; ".join(f"{k} {v}" for k, v in meshBounds.items())
    d, nE, nN = C.c_int(), C.c_int(), C.c_int()
    fn, mb = os.fsencode(fileName), meshBounds.encode()
    _check(lib().frg_read_gmsh(fn, mb, C.byref(d), C.byref(nE), C.byref(nN), None, None, None))
    nd, ne, nn = d.value, nE.value, nN.value
    xv = np.empty((ne, nn, nd), np.float64)
    c2v = np.empty((ne, 4 if nd == 2 else 8), np.int32)
    bc = np.empty((ne, 4 if nd == 2 else 6), np.int32)
    _check(lib().frg_read_gmsh(fn, mb, C.byref(d), C.byref(nE), C.byref(nN), xv.ctypes.data, c2v.ctypes.data,
                               bc.ctypes.data))
    return Mesh(nd, xv, c2v, bc)


class Ensemble:
    """Solvers advanced together, one graph launch per step (frg_ensemble)."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s.h for s in self.solvers])
        h = C.c_void_p()
        _check(lib().frg_ensemble_create(arr, len(self.solvers), C.byref(h)))
        self.h = h

    def set_stream(self, stream_ptr):
        _check(lib().frg_ensemble_set_stream(self.h, stream_ptr))

    def update(self, nsteps=1):
        _check(lib().frg_ensemble_update(self.h, nsteps))

    def close(self):
        if getattr(self, "h", None):
            lib().frg_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
