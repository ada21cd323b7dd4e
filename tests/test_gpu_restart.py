"""Restart through the solver handle (frg_write_paraview / frg_read_restart):
a run stopped, written, and resumed in a new solver continues as the
uninterrupted run does, to the file's 16 significant digits."""
import numpy as np
import pytest

from fr_learn_b200.solver import FRG_MIXED

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, FRG_MIXED])
def test_write_then_restart_continues_the_run(tmp_path, precision):
    from fr_learn_b200 import Solver, box2d

    mesh = box2d(8, 8, -10, 10, -10, 10, perturb=0.1, seed=21)
    kw = dict(order=4, riemannType=1, dtType=1, CFL=0.5, precision=precision)
    base = str(tmp_path / "vortex")
    with Solver(mesh, **kw) as a:
        a.setInitialCondition(1)
        a.update(5)
        a.write_paraview(base)
        U5, t5 = a.get("U_spts"), a.time
        with Solver(mesh, **kw) as b:
            b.read_restart(base, 5)
            assert b.iter == 5 and abs(b.time - t5) <= 1e-15 * t5  # TIME has 16 digits
            assert np.abs(b.get("U_spts") - U5).max() <= 1e-14 * np.abs(U5).max()
            # the uninterrupted run recomputes its wave speeds here too, so the
            # two runs take the same dt path
            a.setIter(5, 5)
            a.update(4)
            b.update(4)
            assert b.iter == 9
            assert abs(b.time - a.time) <= 1e-14 * a.time
            Ua, Ub = a.get("U_spts"), b.get("U_spts")
            assert np.abs(Ua - Ub).max() <= 1e-12 * np.abs(Ua).max()
    with open(f"{base}_{5:09d}.vtu") as f:
        head = f.read(400)
    assert "<!-- ITER 5 -->" in head and f"<!-- TIME {t5:.16g} -->" in head
