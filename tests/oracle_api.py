"""ctypes binding of the CPU oracle (oracle/_ref/liboracle.so) -- test
infrastructure, used only by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, and only as the checker / CPU timing baseline."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")


class OrcParams(C.Structure):
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
        ("wWall", C.c_double),
    ]


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        for f in ("orc_nspts", "orc_nfpts", "orc_nfields", "orc_nfaces", "orc_get_iter"):
            getattr(L, f).argtypes = [C.c_void_p]
            getattr(L, f).restype = C.c_int
        for f in ("orc_get_dt", "orc_get_time"):
            getattr(L, f).argtypes = [C.c_void_p]
            getattr(L, f).restype = C.c_double
        L.orc_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_get.restype = C.c_long
        L.orc_set.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_set.restype = C.c_long
        L.orc_get_faces.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_set_ic.argtypes = [C.c_void_p, C.c_int, C.c_double]
        for f in ("orc_extrapolate_u", "orc_calc_dt", "orc_update"):
            getattr(L, f).argtypes = [C.c_void_p]
        L.orc_calc_residual.argtypes = [C.c_void_p, C.c_int]
        L.orc_time_step_a.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_time_step_b.argtypes = [C.c_void_p, C.c_int]
        L.orc_residual_norm.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_wall_force.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_mass_flux.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_integrate_error.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                          C.c_void_p]
        _lib = L
    return _lib


def params(**kw) -> OrcParams:
    """Defaults follow input::readInputFile (src/input.cpp:214-475)."""
    d = dict(nDims=2, order=3, equation=1, viscous=0, riemannType=0, vcjhScheme=0, timeType=4, dtType=0,
             dt=1e-3, CFL=0.5, gamma=1.4, advectVx=1.0, advectVy=1.0, advectVz=0.0, lambda_=1.0, diffD=1.0,
             rhoBound=1.0, uBound=0.2, vBound=0.0, wBound=0.0, pBound=0.7142857143,
             mu_inf=1.0 / 1600.0, prandtl=0.72, c_sth=0.0, rt_inf=1.0, fixVis=1, penFact=0.0, tau=1.0,
             TWall=1.0, RGas=1.0, uWall=0.0, vWall=0.0, wWall=0.0)
    if "lambda" in kw:
        kw["lambda_"] = kw.pop("lambda")
    d.update(kw)
    return OrcParams(**d)


class Oracle:
    def __init__(self, p: OrcParams, mesh):
        L = lib()
        self.p = p
        self.mesh = mesh
        xv = np.ascontiguousarray(mesh.xv, np.float64)
        c2v = np.ascontiguousarray(mesh.c2v, np.int32)
        bc = np.ascontiguousarray(mesh.bc, np.int32)
        self._keep = (xv, c2v, bc)
        h = L.orc_create(C.byref(p), mesh.nEles, mesh.nNodes, xv.ctypes.data, c2v.ctypes.data, bc.ctypes.data)
        if not h:
            raise RuntimeError("oracle: orc_create failed (see stderr)")
        self.h = h
        self.nS = L.orc_nspts(h)
        self.nF = L.orc_nfpts(h)
        self.nV = L.orc_nfields(h)
        self.nE = mesh.nEles

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get(self, name):
        L = lib()
        n = L.orc_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, np.float64)
        L.orc_get(self.h, name.encode(), out.ctypes.data)
        return out

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, np.float64).ravel()
        n = lib().orc_get(self.h, name.encode(), None)
        assert a.size == n, (name, a.size, n)
        lib().orc_set(self.h, name.encode(), a.ctypes.data)

    def faces(self):
        n = lib().orc_nfaces(self.h)
        out = np.empty((n, 6), np.int32)
        lib().orc_get_faces(self.h, out.ctypes.data)
        return out

    # shaped views, reference layouts
    def U(self):
        return self.get("U_spts").reshape(self.nS, self.nE, self.nV)

    def set_ic(self, ic, a0=0.0):
        lib().orc_set_ic(self.h, ic, a0)

    def calc_residual(self, step=0):
        lib().orc_calc_residual(self.h, step)

    def divF(self, step=0):
        return self.get(f"divF_spts{step}").reshape(self.nS, self.nE, self.nV)

    def update(self, n=1):
        for _ in range(n):
            lib().orc_update(self.h)

    def calc_dt(self):
        lib().orc_calc_dt(self.h)

    @property
    def dt(self):
        return lib().orc_get_dt(self.h)

    @property
    def time(self):
        return lib().orc_get_time(self.h)

    def residual_norm(self, norm_type=2):
        out = np.zeros(self.nV)
        lib().orc_residual_norm(self.h, norm_type, out.ctypes.data)
        return out

    def wall_force(self):
        out = np.zeros(6)
        lib().orc_wall_force(self.h, out.ctypes.data)
        return out

    def mass_flux(self, error_norm=0):
        out = np.zeros(self.nV)
        lib().orc_mass_flux(self.h, error_norm, out.ctypes.data)
        return out

    def integrate_error(self, ic_type, error_norm=1, quad_order=10, box=(-5.0, 5.0, -5.0, 5.0), eps=5.0):
        out = np.zeros(self.nV)
        b = np.ascontiguousarray(box, np.float64)
        lib().orc_integrate_error(self.h, ic_type, eps, error_norm, quad_order, b.ctypes.data, out.ctypes.data)
        return out
