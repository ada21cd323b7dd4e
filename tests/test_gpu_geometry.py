"""Element metrics on the device (frg_update_geometry) against the host set-up.

A solver whose mesh nodes are moved on the device must hold bitwise the
metrics of a solver created on the moved mesh (solver::updateTransforms,
src/solver.cpp:1358-1363, against calcTransforms at set-up, :1227-1356), and
so give bitwise the same residual and the same steps, CFL dt included.
"""
import numpy as np
import pytest

from fr_learn_b200.solver import FRG_MIXED

pytestmark = pytest.mark.gpu


def cases():
    from fr_learn_b200 import box2d, box3d, bump2d

    char6 = {s: "char" for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    return {
        # (mesh before, mesh after, initial condition (icType, a0), solver parameters)
        "quad4_p4_roe_mixed": (box2d(8, 8, -10, 10, -10, 10, perturb=0.1, seed=3),
                               box2d(8, 8, -10, 10, -10, 10, perturb=0.1, seed=4), 1,
                               dict(order=4, riemannType=1, dtType=1, CFL=0.5, precision=FRG_MIXED)),
        "quad4_p3_rusanov_fp64": (box2d(6, 7, -10, 10, -10, 10, perturb=0.05, seed=5),
                                  box2d(6, 7, -10, 10, -10, 10, perturb=0.1, seed=6), 1,
                                  dict(order=3, riemannType=0, dtType=1, CFL=0.5)),
        "quad9_bump_p3_fp64": (bump2d(12, 4), bump2d(12, 4, amp=0.05), 0,
                               dict(order=3, riemannType=1, dtType=1, CFL=0.5, uBound=0.5 * np.sqrt(1.4),
                                    pBound=1.0)),
        "hex8_p3_periodic_fp64": (box3d(3, 3, 4, perturb=0.05, seed=7), box3d(3, 3, 4, perturb=0.1, seed=8), (10, 0.1),
                                  dict(order=3, dtType=1, CFL=0.25)),
        "hex8_p2_char_mixed": (box3d(3, 3, 3, (-2, -2, -2), (2, 2, 2), bcs=char6, perturb=0.1, seed=1),
                               box3d(3, 3, 3, (-2, -2, -2), (2, 2, 2), bcs=char6, perturb=0.1, seed=2), 1,
                               dict(order=2, dtType=1, CFL=0.5, precision=FRG_MIXED)),
    }


CASES = cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_metrics_match_host_setup(name):
    from fr_learn_b200 import Solver

    meshA, meshB, ic, kw = CASES[name]
    ic = ic if isinstance(ic, tuple) else (ic, 0.0)
    assert np.array_equal(meshA.c2v, meshB.c2v) and np.array_equal(meshA.bc, meshB.bc)
    with Solver(meshA, **kw) as gA, Solver(meshB, **kw) as gB:
        gA.setInitialCondition(*ic)
        gA.update(2)  # a solver mid-run: its next dt must see the new normals
        before = gA.launch_count()
        gA.update_geometry(meshB.xv)
        assert gA.launch_count() - before == 3
        assert np.array_equal(gA.get("detJac_spts"), gB.get("detJac_spts"))
        assert np.array_equal(gA.get("pos_spts"), gB.get("pos_spts"))
        gB.setInitialCondition(*ic)
        U = gB.get("U_spts")
        gA.set("U_spts", U)
        gA.calcResidual(0)
        gB.calcResidual(0)
        assert np.array_equal(gA.get("divF_spts"), gB.get("divF_spts"))
        gA.update(3)
        gB.update(3)
        assert gA.dt == gB.dt
        assert np.array_equal(gA.get("U_spts"), gB.get("U_spts"))
        assert not np.array_equal(gA.get("U_spts"), U)


def test_negative_jacobian_leaves_metrics_unchanged():
    from fr_learn_b200 import Solver, box2d
    from fr_learn_b200.solver import FrgError

    mesh = box2d(6, 6, -10, 10, -10, 10, perturb=0.1, seed=11)
    with Solver(mesh, order=3, dtType=0, dt=1e-3) as g:
        g.setInitialCondition(1)
        g.calcResidual(0)
        det0, div0 = g.get("detJac_spts"), g.get("divF_spts")
        bad = mesh.xv.copy()
        bad[4, :, 0] *= -1.0  # mirror one element: negative Jacobian
        with pytest.raises(FrgError) as ei:
            g.update_geometry(bad)
        assert ei.value.code == 4 and "element 4" in str(ei.value)
        assert np.array_equal(g.get("detJac_spts"), det0)
        g.calcResidual(0)
        assert np.array_equal(g.get("divF_spts"), div0)
        # the same nodes again: nothing moves
        g.update_geometry(mesh.xv)
        g.calcResidual(0)
        assert np.array_equal(g.get("divF_spts"), div0)
