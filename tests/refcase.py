"""Drive the FlurryPP reference harness (oracle/_ref/refharness) -- test
infrastructure for generating golden fixtures in the container that has the
reference sources.  Writes a Gmsh v2 hexahedral mesh and a reference input
file for a box mesh from fr_learn_b200.mesh, runs the harness and loads the
arrays it dumps."""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "refharness")
BCNAME = {1: "char", 2: "sup_in", 3: "sup_out", 4: "sub_in", 5: "sub_out", 8: "slip_wall",
          9: "isothermal_noslip", 10: "adiabatic_noslip"}
HEXFV = ((0, 1, 2, 3), (4, 5, 6, 7), (3, 0, 4, 7), (2, 1, 5, 6), (1, 0, 4, 5), (3, 2, 6, 7))
# the reference checkout whose sources oracle/Makefile compiles
REFDIR = os.environ.get("REFDIR", "/root/reference")


def available() -> bool:
    return os.path.isdir(os.path.join(REFDIR, "src"))


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REFDIR={REFDIR}"], check=True)


def load(outdir):
    res = {}
    with open(os.path.join(outdir, "manifest.txt")) as f:
        for line in f:
            parts = line.split()
            name, dt, dims = parts[0], parts[1], [int(x) for x in parts[2:]]
            a = np.fromfile(os.path.join(outdir, f"{name}.{dt}"), dtype=np.float64 if dt == "f64" else np.int32)
            res[name] = a.reshape(dims)
    return res


def write_gmsh(mesh, path):
    """Gmsh v2 ASCII file of a (non-periodic) 8-node hex mesh."""
    assert mesh.nDims == 3 and mesh.nNodes == 8
    verts = mesh.verts
    names = sorted({int(b) for b in mesh.bc.ravel() if b >= 0})
    phys = {b: i + 1 for i, b in enumerate(names)}
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(names) + 1)]
    for b in names:
        lines.append(f'2 {phys[b]} "{BCNAME[b]}"')
    lines.append('3 99 "fluid"')
    lines += ["$EndPhysicalNames", "$Nodes", str(len(verts))]
    for i, v in enumerate(verts):
        lines.append(f"{i + 1} {v[0]:.17g} {v[1]:.17g} {v[2]:.17g}")
    lines += ["$EndNodes", "$Elements"]
    els = []
    for e in range(mesh.nEles):
        for f in range(6):
            b = int(mesh.bc[e, f])
            if b >= 0:
                vs = [int(mesh.c2v[e, k]) + 1 for k in HEXFV[f]]
                els.append(f"3 2 {phys[b]} {phys[b]} " + " ".join(map(str, vs)))
    for e in range(mesh.nEles):
        els.append("5 2 99 99 " + " ".join(str(int(v) + 1) for v in mesh.c2v[e]))
    lines.append(str(len(els)))
    lines += [f"{i + 1} {s}" for i, s in enumerate(els)]
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return {BCNAME[b] for b in names}


def write_input(path, mesh_file, bcnames, **kw):
    opts = dict(equation=1, nDims=3, icType=1, order=2, timeType=4, dtType=0, dt=1e-3, CFL=0.5,
                iterMax=1000000, maxTime=1e9, viscous=0, riemannType=0, meshType=0,
                gamma=1.4, rhoBound=1.0, uBound=0.2, vBound=0.0, wBound=0.0, pBound=0.7142857143,
                monitorResFreq=1000000, plotFreq=1000000, restart=0)
    opts.update(kw)
    with open(path, "w") as f:
        for k, v in opts.items():
            f.write(f"{k} {v!r}\n" if isinstance(v, float) else f"{k} {v}\n")
        f.write(f"meshFileName {mesh_file}\n")
        for b in bcnames:
            f.write(f"mesh_bound {b} {b}\n")
        f.write("mesh_bound fluid fluid\n")


def run_case(mesh, nsteps=0, workdir=None, **kw):
    """Run the harness 'case' mode; returns the dumped arrays."""
    if not os.path.exists(HARNESS):
        build()
    wd = workdir or tempfile.mkdtemp(prefix="frref_")
    msh = os.path.join(wd, "mesh.msh")
    bcnames = write_gmsh(mesh, msh)
    inp = os.path.join(wd, "input.txt")
    write_input(inp, msh, bcnames, **kw)
    out = os.path.join(wd, "out")
    subprocess.run([HARNESS, "case", inp, out, str(nsteps)], check=True, cwd=wd,
                   stdout=subprocess.DEVNULL)
    return load(out)


def run_vtu(mesh, nsteps=0, workdir=None, **kw):
    """Run the harness 'vtu' mode: the dumped arrays plus the text of the
    ParaView / restart file the reference wrote."""
    if not os.path.exists(HARNESS):
        build()
    wd = workdir or tempfile.mkdtemp(prefix="frref_")
    msh = os.path.join(wd, "mesh.msh")
    bcnames = write_gmsh(mesh, msh)
    inp = os.path.join(wd, "input.txt")
    write_input(inp, msh, bcnames, **kw)
    out = os.path.join(wd, "out")
    subprocess.run([HARNESS, "vtu", inp, out, str(nsteps)], check=True, cwd=wd, stdout=subprocess.DEVNULL)
    res = load(out)
    it = int(res["iter"][0])
    with open(os.path.join(out, f"ref_{it:09d}.vtu")) as f:
        res["vtu"] = f.read()
    return res


def run_ops(nDims, order, vcjh=0):
    if not os.path.exists(HARNESS):
        build()
    out = tempfile.mkdtemp(prefix="frops_")
    subprocess.run([HARNESS, "ops", str(nDims), str(order), str(vcjh), out], check=True,
                   stdout=subprocess.DEVNULL)
    return load(out)


def run_kat():
    if not os.path.exists(HARNESS):
        build()
    out = tempfile.mkdtemp(prefix="frkat_")
    subprocess.run([HARNESS, "kat", out], check=True, stdout=subprocess.DEVNULL)
    return load(out)


def run_integrals(mesh, nsteps=0, workdir=None, **kw):
    """Run the harness 'integrals' mode: the state after nsteps updates and
    the reference's computeWallForce / computeMassFlux / integrateError."""
    if not os.path.exists(HARNESS):
        build()
    wd = workdir or tempfile.mkdtemp(prefix="frref_")
    msh = os.path.join(wd, "mesh.msh")
    bcnames = write_gmsh(mesh, msh)
    inp = os.path.join(wd, "input.txt")
    write_input(inp, msh, bcnames, **kw)
    out = os.path.join(wd, "out")
    subprocess.run([HARNESS, "integrals", inp, out, str(nsteps)], check=True, cwd=wd, stdout=subprocess.DEVNULL)
    return load(out)
