"""The reference-side binding (fr_learn_b200/shim/solver_gpu.cpp, shown in
INTEGRATION.md) compiles against the reference's own headers and links with
the reference's objects and libfrgpu.so.  CPU only; needs the reference
sources (skipped where they are absent).  The linked program reads a
reference input file and converts it with frgpu_params; frgpu_setup and
frgpu_update need a GPU and are exercised on one through the same C ABI by
the other tests."""
import glob
import os
import subprocess

import pytest

import refcase

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MAIN = r'''
#include <cstdio>
#include "frgpu.h"
#include "input.hpp"
frg_params frgpu_params(const input *p);
int main(int argc, char **argv) {
  input params;
  params.rank = 0;
  params.nproc = 1;
  params.readInputFile(argv[1]);
  frg_params q = frgpu_params(&params);
  printf("%d %d %d %d %d %.17g %.17g\n", q.nDims, q.order, q.equation, q.vcjhScheme, q.timeType, q.CFL, q.gamma);
  return 0;
}
'''


@pytest.mark.skipif(not refcase.available(), reason="reference sources not present")
def test_shim_compiles_and_links_against_reference(tmp_path):
    refcase.build()  # the reference's objects (oracle/_ref/refobj)
    inc = os.path.join(refcase.REFDIR, "include")
    objs = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "refobj", "*.o")))
    assert objs
    main = tmp_path / "main.cpp"
    main.write_text(MAIN)
    exe = str(tmp_path / "shimtest")
    flags = ["-std=c++11", "-O1", "-w", f"-I{inc}", f"-I{os.path.join(ROOT, 'include')}",
             f"-I{os.path.join(ROOT, 'oracle', 'refshim')}"]
    shim = os.path.join(ROOT, "fr_learn_b200", "shim", "solver_gpu.cpp")
    libdir = os.path.join(ROOT, "fr_learn_b200")
    cmd = ["g++"] + flags + [shim, str(main)] + objs + [f"-L{libdir}", "-lfrgpu", f"-Wl,-rpath,{libdir}",
                                                         "-lpthread", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    # a reference input file: its parameters come through frgpu_params
    from fr_learn_b200 import box3d

    mesh = box3d(2, 2, 2, (-1, -1, -1), (1, 1, 1),
                 bcs={s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")})
    msh = str(tmp_path / "m.msh")
    names = refcase.write_gmsh(mesh, msh)
    inp = str(tmp_path / "input.txt")
    refcase.write_input(inp, msh, names, order=3, timeType=4, dtType=1, CFL=0.3, vcjhSchemeQuad=2)
    out = subprocess.run([exe, inp], capture_output=True, text=True, cwd=str(tmp_path))
    assert out.returncode == 0, out.stderr
    vals = out.stdout.split()[-7:]
    assert vals[:5] == ["3", "3", "1", "2", "4"]
    assert float(vals[5]) == 0.3 and float(vals[6]) == 1.4
