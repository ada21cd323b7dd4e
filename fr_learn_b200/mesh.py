"""Structured quad / hex mesh generators for the FR path (host side, setup only).

The reference reads Gmsh v2 hexahedra (src/geo.cpp:448-769) and matches faces
by sorted vertex lists (src/geo.cpp:75-246); it has no periodic pairing and no
2D reader.  These generators produce what the solver needs directly:

* ``xv``  [nEles][nNodes][nDims]  element node coordinates in the reference's
  shape-node order (Gmsh order: corners counter-clockwise, then edge
  mid-nodes bottom/right/top/left, then the centre node, src/funcs.cpp:126-176);
* ``c2v`` [nEles][nCorners]  vertex ids used only for face matching.  Periodic
  images share one id, so the reference's own matching and orientation rules
  (src/geo.cpp:789-908) pair periodic faces;
* ``bc``  [nEles][nFacesPerEle]  boundary-condition code (the reference's
  BC_TYPE, include/global.hpp:63-78) of element faces on a non-periodic
  boundary, -1 elsewhere.

Element faces follow the reference's local numbering: QUAD 0 bottom (eta=-1),
1 right, 2 top, 3 left; HEX 0 zmin, 1 zmax, 2 xmin, 3 xmax, 4 ymin, 5 ymax
(src/geo.cpp:85-90).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# BC_TYPE of include/global.hpp:63-78
BC = {
    "periodic": 0,
    "char": 1,
    "sup_in": 2,
    "sup_out": 3,
    "sub_in": 4,
    "sub_out": 5,
    "slip_wall": 8,
    "isothermal_noslip": 9,
    "adiabatic_noslip": 10,
    "symmetry": 12,
    "none": -1,
}


@dataclass
class Mesh:
    nDims: int
    xv: np.ndarray  # [nE][nN][d] float64
    c2v: np.ndarray  # [nE][nC] int32
    bc: np.ndarray  # [nE][nFaceEle] int32
    # unique vertex coordinates for c2v ids (periodic images collapsed)
    verts: np.ndarray = field(default=None)
    name: str = ""

    @property
    def nEles(self) -> int:
        return self.xv.shape[0]

    @property
    def nNodes(self) -> int:
        return self.xv.shape[1]


def _perturbation(rng, shape, amp):
    return rng.uniform(-amp, amp, size=shape)


def box2d(nx, ny, x0=-5.0, x1=5.0, y0=-5.0, y1=5.0, bcs=None, perturb=0.0, seed=0):
    """Linear quads on [x0,x1]x[y0,y1].

    ``bcs`` maps 'xmin','xmax','ymin','ymax' to a BC name; missing sides are
    periodic (both sides of a direction must agree).  ``perturb`` moves every
    vertex by a seeded uniform amount in +-perturb*h per coordinate, except the
    boundary-normal coordinate of vertices on non-periodic sides; periodic
    images move together.
    """
    bcs = dict(bcs or {})
    per = {
        0: bcs.get("xmin", "periodic") == "periodic",
        1: bcs.get("ymin", "periodic") == "periodic",
    }
    if per[0] != (bcs.get("xmax", "periodic") == "periodic") or per[1] != (bcs.get("ymax", "periodic") == "periodic"):
        raise ValueError("a direction is periodic on one side only")
    n = (nx, ny)
    # with 2 elements across a periodic direction both neighbours share all
    # vertex ids, so vertex-based face matching would be ambiguous
    if (per[0] and nx < 3) or (per[1] and ny < 3):
        raise ValueError("periodic directions need at least 3 elements")
    h = ((x1 - x0) / nx, (y1 - y0) / ny)
    L = (x1 - x0, y1 - y0)
    rng = np.random.default_rng(seed)
    # canonical vertex lattice (periodic directions have n vertices, else n+1)
    nvx, nvy = (nx if per[0] else nx + 1), (ny if per[1] else ny + 1)
    I, J = np.meshgrid(np.arange(nvx), np.arange(nvy), indexing="ij")
    base = np.stack([x0 + I * h[0], y0 + J * h[1]], axis=-1).astype(np.float64)
    if perturb > 0:
        dx = _perturbation(rng, base.shape, perturb * np.array(h))
        if not per[0]:
            dx[0, :, 0] = 0
            dx[-1, :, 0] = 0
        if not per[1]:
            dx[:, 0, 1] = 0
            dx[:, -1, 1] = 0
        base = base + dx
    vid = (I * nvy + J).astype(np.int64)

    def vert(i, j):
        """(id, coordinates) of lattice vertex (i, j), unwrapping periodic images."""
        oi, oj = 0.0, 0.0
        ii, jj = i, j
        if per[0] and i == nx:
            ii, oi = 0, L[0]
        if per[1] and j == ny:
            jj, oj = 0, L[1]
        return vid[ii, jj], base[ii, jj] + np.array([oi, oj])

    nE = nx * ny
    xv = np.zeros((nE, 4, 2))
    c2v = np.zeros((nE, 4), np.int32)
    bc = -np.ones((nE, 4), np.int32)
    e = 0
    for j in range(ny):
        for i in range(nx):
            for k, (a, b) in enumerate(((i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1))):
                c2v[e, k], xv[e, k] = vert(a, b)
            if j == 0 and not per[1]:
                bc[e, 0] = BC[bcs["ymin"]]
            if i == nx - 1 and not per[0]:
                bc[e, 1] = BC[bcs["xmax"]]
            if j == ny - 1 and not per[1]:
                bc[e, 2] = BC[bcs["ymax"]]
            if i == 0 and not per[0]:
                bc[e, 3] = BC[bcs["xmin"]]
            e += 1
    return Mesh(2, xv, c2v, bc, verts=base.reshape(-1, 2), name=f"box2d_{nx}x{ny}")


def box3d(nx, ny, nz, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), bcs=None, perturb=0.0, seed=0):
    """Linear (8-node) hexahedra on a box; same conventions as :func:`box2d`
    with sides 'xmin','xmax','ymin','ymax','zmin','zmax'."""
    bcs = dict(bcs or {})
    names = (("xmin", "xmax"), ("ymin", "ymax"), ("zmin", "zmax"))
    per = {}
    for d, (a, b) in enumerate(names):
        pa, pb = bcs.get(a, "periodic") == "periodic", bcs.get(b, "periodic") == "periodic"
        if pa != pb:
            raise ValueError("a direction is periodic on one side only")
        per[d] = pa
    n = (nx, ny, nz)
    for d in range(3):
        if per[d] and n[d] < 3:
            raise ValueError("periodic directions need at least 3 elements")
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    L = hi - lo
    h = L / np.array(n)
    nv = [n[d] if per[d] else n[d] + 1 for d in range(3)]
    I, J, K = np.meshgrid(np.arange(nv[0]), np.arange(nv[1]), np.arange(nv[2]), indexing="ij")
    base = np.stack([lo[0] + I * h[0], lo[1] + J * h[1], lo[2] + K * h[2]], axis=-1)
    if perturb > 0:
        rng = np.random.default_rng(seed)
        dx = _perturbation(rng, base.shape, perturb * h)
        for d in range(3):
            if not per[d]:
                sl = [slice(None)] * 3
                sl[d] = 0
                dx[tuple(sl) + (d,)] = 0
                sl[d] = -1
                dx[tuple(sl) + (d,)] = 0
        base = base + dx
    vid = (I * nv[1] * nv[2] + J * nv[2] + K).astype(np.int64)

    def vert(i, j, k):
        idx = [i, j, k]
        off = np.zeros(3)
        for d in range(3):
            if per[d] and idx[d] == n[d]:
                idx[d] = 0
                off[d] = L[d]
        return vid[idx[0], idx[1], idx[2]], base[idx[0], idx[1], idx[2]] + off

    nE = nx * ny * nz
    xv = np.zeros((nE, 8, 3))
    c2v = np.zeros((nE, 8), np.int32)
    bc = -np.ones((nE, 6), np.int32)
    corners = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))
    e = 0
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for c, (a, b, g) in enumerate(corners):
                    c2v[e, c], xv[e, c] = vert(i + a, j + b, k + g)
                if k == 0 and not per[2]:
                    bc[e, 0] = BC[bcs["zmin"]]
                if k == nz - 1 and not per[2]:
                    bc[e, 1] = BC[bcs["zmax"]]
                if i == 0 and not per[0]:
                    bc[e, 2] = BC[bcs["xmin"]]
                if i == nx - 1 and not per[0]:
                    bc[e, 3] = BC[bcs["xmax"]]
                if j == 0 and not per[1]:
                    bc[e, 4] = BC[bcs["ymin"]]
                if j == ny - 1 and not per[1]:
                    bc[e, 5] = BC[bcs["ymax"]]
                e += 1
    return Mesh(3, xv, c2v, bc, verts=base.reshape(-1, 3), name=f"box3d_{nx}x{ny}x{nz}")


def bump2d(nx=96, ny=32, x0=-1.5, x1=1.5, height=0.8, amp=0.0625, width=25.0, cluster=1.5,
           bc_in="char", bc_out="char", bc_wall="slip_wall", bc_top=None):
    """Channel over a Gaussian bump with 9-node (quadratic) quads.

    Lower wall y_w(x) = amp*exp(-width*x^2), upper wall y = height.  Points are
    mapped algebraically, y = y_w(x) + (height - y_w(x)) * s(eta), with the
    wall-clustering stretch s(eta) = 1 + tanh(c(eta-1))/tanh(c), eta in [0,1].
    Inlet (xmin) / outlet (xmax) take ``bc_in`` / ``bc_out``; the lower wall
    ``bc_wall``, the upper one ``bc_top`` (default: ``bc_wall``; "symmetry"
    gives the same ghost state but keeps it out of wall integrals).
    """
    bc_top = bc_wall if bc_top is None else bc_top
    X = np.linspace(x0, x1, 2 * nx + 1)
    eta = np.linspace(0.0, 1.0, 2 * ny + 1)
    s = 1.0 + np.tanh(cluster * (eta - 1.0)) / np.tanh(cluster)
    yw = amp * np.exp(-width * X ** 2)
    PX = np.repeat(X[:, None], 2 * ny + 1, axis=1)
    PY = yw[:, None] + (height - yw[:, None]) * s[None, :]
    pid = np.arange((2 * nx + 1) * (2 * ny + 1)).reshape(2 * nx + 1, 2 * ny + 1)
    nE = nx * ny
    xv = np.zeros((nE, 9, 2))
    c2v = np.zeros((nE, 4), np.int32)
    bc = -np.ones((nE, 4), np.int32)
    # node (a,b) offsets in the 3x3 point block, shape_quad order
    order = ((0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1))
    e = 0
    for j in range(ny):
        for i in range(nx):
            for k, (a, b) in enumerate(order):
                xv[e, k] = (PX[2 * i + a, 2 * j + b], PY[2 * i + a, 2 * j + b])
            for k, (a, b) in enumerate(order[:4]):
                c2v[e, k] = pid[2 * i + a, 2 * j + b]
            if j == 0:
                bc[e, 0] = BC[bc_wall]
            if i == nx - 1:
                bc[e, 1] = BC[bc_out]
            if j == ny - 1:
                bc[e, 2] = BC[bc_top]
            if i == 0:
                bc[e, 3] = BC[bc_in]
            e += 1
    verts = np.stack([PX.ravel(), PY.ravel()], axis=-1)
    return Mesh(2, xv, c2v, bc, verts=verts, name=f"bump2d_{nx}x{ny}")


def concat_meshes(meshes):
    """One mesh holding independent cases side by side (for the ensemble
    mode): element arrays stacked, vertex ids offset per case so no face joins
    two cases.  Returns (mesh, group of each element)."""
    assert meshes and all(m.nDims == meshes[0].nDims and m.nNodes == meshes[0].nNodes for m in meshes)
    xv, c2v, bc, verts, grp = [], [], [], [], []
    off = 0
    for g, m in enumerate(meshes):
        nv = int(m.c2v.max()) + 1 if m.verts is None else len(m.verts)
        xv.append(m.xv)
        c2v.append(m.c2v + off)
        bc.append(m.bc)
        if m.verts is not None:
            verts.append(m.verts)
        grp.append(np.full(m.nEles, g, np.int32))
        off += nv
    out = Mesh(meshes[0].nDims, np.concatenate(xv), np.concatenate(c2v).astype(np.int32), np.concatenate(bc),
               verts=np.concatenate(verts) if len(verts) == len(meshes) else None,
               name=f"ensemble_{len(meshes)}")
    return out, np.concatenate(grp)
