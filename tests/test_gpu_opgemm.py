"""Tensor-core operator GEMMs (frg_apply_operator): the oper::apply* products
(src/operators.cpp:1191-1450) as 3xTF32 tcgen05 GEMMs, checked against the
dense FP64 operator applied on the host.

Bar: max |Y - Y_ref| <= 1e-5 * max |Y_ref| (3xTF32 split precision, FP32
accumulation), for every operator, dimension and field; columns beyond
nEles are left untouched.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def solver_for(case):
    import torch

    from fr_learn_b200 import FRG_MIXED, Solver, box2d, box3d

    if case == "quad_p4":
        s = Solver(box2d(13, 11, perturb=0.1, seed=3), order=4, precision=FRG_MIXED)
    elif case == "quad_p2":
        s = Solver(box2d(5, 7), order=2, precision=FRG_MIXED)
    elif case == "hex_p3":
        s = Solver(box3d(6, 5, 7, perturb=0.1, seed=4), order=3, viscous=1, precision=FRG_MIXED)
    else:
        raise ValueError(case)
    # the arrays are produced on torch's stream: run the kernel there too
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    return s


def shapes(s, which):
    nS, nF = s.nSpts, s.nFpts
    return {0: (nF, nS), 1: (nS, nS), 2: (nF, nS), 3: (nS, nF), 4: (nS, nF)}[which]


@pytest.mark.parametrize("case", ["quad_p4", "quad_p2", "hex_p3"])
@pytest.mark.parametrize("which", [0, 1, 2, 3, 4])
def test_apply_operator_matches_dense_fp64(case, which):
    import torch

    s = solver_for(case)
    nV, nE = s.nFields, s.nEles
    ld = (nE + 31) // 32 * 32 + 32  # a padded stride, with columns beyond nEles
    M, K = shapes(s, which)
    g = torch.Generator().manual_seed(100 * which + len(case))
    dims = range(s.params["nDims"]) if which in (1, 2, 4) else [0]
    for dim in dims:
        op = s.operator(which, dim)
        assert op.shape == (M, K)
        X = torch.randn((nV, K, ld), generator=g, dtype=torch.float32)
        Y0 = torch.randn((nV, M, ld), generator=g, dtype=torch.float32)
        for beta in (0.0, 1.0, -0.5):
            Xd, Yd = X.cuda(), Y0.cuda()
            s.apply_operator(which, dim, Xd.data_ptr(), Yd.data_ptr(), ld, beta)
            s.sync()
            Y = Yd.cpu().numpy().astype(np.float64)
            Xn, Yn = X.numpy().astype(np.float64), Y0.numpy().astype(np.float64)
            ref = np.einsum("mk,vke->vme", op, Xn[:, :, :nE]) + beta * Yn[:, :, :nE]
            err = np.abs(Y[:, :, :nE] - ref).max() / np.abs(ref).max()
            assert err <= TOL, (case, which, dim, beta, err)
            assert np.array_equal(Y[:, :, nE:], Yn[:, :, nE:])  # padding columns not written
    s.set_stream(None)


def test_apply_operator_is_more_accurate_than_tf32():
    """The split-precision products carry FP32-level accuracy: one TF32
    product would be off by ~1e-3 relative."""
    import torch

    s = solver_for("hex_p3")
    nV, nE = s.nFields, s.nEles
    ld = (nE + 31) // 32 * 32
    op = s.operator(1, 2)
    X = torch.rand((nV, s.nSpts, ld), dtype=torch.float32) + 1.0
    Xd = X.cuda()
    Yd = torch.zeros((nV, s.nSpts, ld), dtype=torch.float32, device="cuda")
    s.apply_operator(1, 2, Xd.data_ptr(), Yd.data_ptr(), ld)
    s.sync()
    ref = np.einsum("mk,vke->vme", op, X.numpy().astype(np.float64)[:, :, :nE])
    err = np.abs(Yd.cpu().numpy()[:, :, :nE] - ref).max() / np.abs(ref).max()
    s.set_stream(None)
    assert err < 2e-6, err


def test_apply_operator_rejects_bad_calls():
    import torch

    from fr_learn_b200 import FRG_MIXED, FrgError, Solver, box3d

    s = solver_for("quad_p2")
    X = torch.zeros((s.nFields, s.nSpts, 64), dtype=torch.float32, device="cuda")
    Y = torch.zeros((s.nFields, s.nFpts, 64), dtype=torch.float32, device="cuda")
    with pytest.raises(FrgError):
        s.apply_operator(5, 0, X.data_ptr(), Y.data_ptr(), 64)
    with pytest.raises(FrgError):
        s.apply_operator(1, 2, X.data_ptr(), Y.data_ptr(), 64)  # a 2D handle has dims 0 and 1
    with pytest.raises(FrgError):
        s.apply_operator(0, 0, X.data_ptr(), Y.data_ptr(), 30)  # stride below nEles / not a multiple of 4
    s.set_stream(None)
    big = Solver(box3d(3, 3, 3), order=4, precision=FRG_MIXED)  # 125 x 150 points: too large for one pass
    X2 = torch.zeros((5, big.nSpts, 32), dtype=torch.float32, device="cuda")
    Y2 = torch.zeros((5, big.nFpts, 32), dtype=torch.float32, device="cuda")
    with pytest.raises(FrgError):
        big.apply_operator(0, 0, X2.data_ptr(), Y2.data_ptr(), 32)


@pytest.mark.parametrize("which", [0, 3])
def test_apply_operator_many_tiles_per_block(which):
    """A mesh large enough that every persistent block takes ~9 tiles: the
    ring of landing slots wraps twice and both TMEM accumulators are reused
    several times (the small meshes above give each block one tile).  300 x
    300 quads, P = 4 (90,000 elements, 2,816 tiles of 128 elements x field),
    plain and accumulating products."""
    import torch

    from fr_learn_b200 import FRG_MIXED, Solver, box2d

    s = Solver(box2d(300, 300), order=4, precision=FRG_MIXED)
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    nV, nE = s.nFields, s.nEles
    ld = (nE + 31) // 32 * 32
    M, K = shapes(s, which)
    op = s.operator(which, 0)
    g = torch.Generator().manual_seed(7 + which)
    X = torch.randn((nV, K, ld), generator=g, dtype=torch.float32)
    Y0 = torch.randn((nV, M, ld), generator=g, dtype=torch.float32)
    Xn = X.numpy().astype(np.float64)[:, :, :nE]
    base = np.einsum("mk,vke->vme", op, Xn)
    for beta in (0.0, 1.0):
        Xd, Yd = X.cuda(), Y0.cuda()
        for _ in range(2):  # two launches in a row, Y reset before each
            Yd.copy_(Y0.cuda())
            s.apply_operator(which, 0, Xd.data_ptr(), Yd.data_ptr(), ld, beta)
        s.sync()
        ref = base + beta * Y0.numpy().astype(np.float64)[:, :, :nE]
        err = np.abs(Yd.cpu().numpy().astype(np.float64)[:, :, :nE] - ref).max() / np.abs(ref).max()
        assert err <= TOL, (which, beta, err)
    s.set_stream(None)
