"""Treecode farfield against the direct farfield (reference:
tests/fmm/test_taylor.py:12-70 -- 20 x 20 rectangles, quad order 2, mac 2.5,
two triangles per leaf, order 8, FP64, agreement to 5 decimals)."""
import numpy as np
import pytest

from tectosaur_b200.fmm.tsfmm import TSFMM, FMMFarfieldOp
from tectosaur_b200.mesh.mesh_gen import concat_no_dedupe, make_rect
from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
from tectosaur_b200.ops.sparse_integral_op import RegularizedSparseIntegralOp

pytestmark = pytest.mark.gpu

CORNERS = [[-1.0, -1.0, 0], [-1.0, 1.0, 0], [1.0, 1.0, 0], [1.0, -1.0, 0]]
TREECODE_KERNELS = ["elasticU3", "elasticRT3", "elasticRA3", "elasticRH3"]


def fmm_case(K_name, float_type=np.float64, offset=0.0, order=8, ppc=2, n=20, seed=123987,
             mode="treecode", mac=2.5):
    rng = np.random.default_rng(seed)
    params = np.array([1.0, 0.25])
    m_src = make_rect(n, n, CORNERS)
    m_obs = make_rect(n, n, CORNERS)
    m_obs[0][:, 0] += offset
    v = rng.random(m_src[1].shape[0] * 9)
    full = concat_no_dedupe(m_src, m_obs)
    src_subset = np.arange(m_src[1].shape[0])
    obs_subset = np.arange(m_obs[1].shape[0]) + m_src[1].shape[0]
    direct = TriToTriDirectFarfieldOp(2, K_name, params, full[0], full[1], float_type,
                                      obs_subset, src_subset)
    y1 = direct.dot(v.astype(float_type))
    fmm = TSFMM(m_obs, m_src, params, order, 2, float_type, K_name, mac, ppc, mode)
    y2 = fmm.dot(v.astype(float_type))
    return fmm, y1, y2


@pytest.mark.parametrize("K", TREECODE_KERNELS)
def test_treecode_matches_direct_fp64(cuda, K):
    fmm, y1, y2 = fmm_case(K)
    assert fmm.m2p.src_n_idxs.shape[0] > 0 and fmm.p2p.src_n_idxs.shape[0] > 0
    np.testing.assert_almost_equal(y1, y2, 5)
    assert np.linalg.norm(y1 - y2) / np.linalg.norm(y1) < 1e-5


@pytest.mark.parametrize("K", ["elasticU3", "elasticRH3"])
def test_treecode_far_only(cuda, K):
    # offset surfaces: every interaction is an M2P
    fmm, y1, y2 = fmm_case(K, offset=6.0)
    assert fmm.p2p.src_n_idxs.shape[0] == 0
    np.testing.assert_almost_equal(y1, y2, 7)


@pytest.mark.parametrize("mode", ["treecode", "fmm"])
def test_error_falls_with_order(cuda, mode):
    errs = []
    for order in [2, 4, 6, 8, 10]:
        _, y1, y2 = fmm_case("elasticRH3", order=order, mode=mode, ppc=4)
        errs.append(np.linalg.norm(y1 - y2) / np.linalg.norm(y1))
    assert all(b < a for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-6, errs


@pytest.mark.parametrize("K", TREECODE_KERNELS)
def test_fmm_mode_matches_direct_fp64(cuda, K):
    fmm, y1, y2 = fmm_case(K, mode="fmm", ppc=4)
    assert fmm.m2l.src_n_idxs.shape[0] > 0 and fmm.p2p.src_n_idxs.shape[0] > 0
    assert np.linalg.norm(y1 - y2) / np.linalg.norm(y1) < 1e-5


@pytest.mark.parametrize("K", ["elasticU3", "elasticRA3", "elasticRH3"])
def test_fmm_mode_fp32(cuda, K):
    _, y1, y2 = fmm_case(K, float_type=np.float32, order=6, mode="fmm", ppc=4)
    assert np.linalg.norm(y1 - y2) / np.linalg.norm(y1) < 1e-4


def test_fmm_mode_high_order_fp32_in_range(cuda):
    # order 12 with small leaves: the radius-scaled expansions stay finite in FP32
    _, y1, y2 = fmm_case("elasticRH3", float_type=np.float32, order=12, mode="fmm", ppc=1, n=24)
    assert np.all(np.isfinite(y2))
    assert np.linalg.norm(y1 - y2) / np.linalg.norm(y1) < 2e-5


@pytest.mark.parametrize("K", ["elasticU3", "elasticRT3", "elasticRA3", "elasticRH3"])
def test_treecode_fp32(cuda, K):
    _, y1, y2 = fmm_case(K, float_type=np.float32, order=6)
    assert np.linalg.norm(y1 - y2) / np.linalg.norm(y1) < 1e-4


def test_treecode_one_leaf_is_direct(cuda):
    # a single leaf holding every triangle: P2P only, equal to the direct sum
    fmm, y1, y2 = fmm_case("elasticRH3", ppc=10 ** 9)
    assert fmm.m2p.src_n_idxs.shape[0] == 0
    assert np.linalg.norm(y1 - y2) / np.linalg.norm(y1) < 1e-12


@pytest.mark.parametrize("mode", ["treecode", "fmm"])
def test_fmm_farfield_op_in_sparse_op(cuda, mode):
    """RegularizedSparseIntegralOp with farfield_op_type = FMMFarfieldOp agrees
    with the direct-farfield operator (the reference's fmm path of
    ops/sparse_integral_op.py)."""
    n = 14
    pts, tris = make_rect(n, n, CORNERS)
    pts = pts.copy()
    pts[:, 2] = 0.1 * np.sin(2 * pts[:, 0]) * np.cos(pts[:, 1])
    pts[:, :2] += 2.0  # positive coordinates, so the max(pts) scaling is used
    args = (6, 6, 5, 2, 4, 2.5, "elasticRH3", "elasticRH3", [1.0, 0.25], pts, tris, np.float64)
    direct = RegularizedSparseIntegralOp(*args, farfield_op_type=TriToTriDirectFarfieldOp)
    fmm = RegularizedSparseIntegralOp(*args, farfield_op_type=FMMFarfieldOp(2.5, 8, 8, mode))
    v = np.random.default_rng(5).random(tris.shape[0] * 9)
    a = direct.dot(v)
    b = fmm.dot(v)
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-5


@pytest.mark.parametrize("float_type", [np.float32, np.float64])
def test_nearfield_overlap_path(cuda, float_type, monkeypatch):
    """Large FMM operators run the nearfield BSR on a second stream next to the
    FMM and add it at the end; forced on a small operator, the single apply,
    the panel apply and a captured graph equal the sequential apply."""
    torch = cuda
    n = 12
    pts, tris = make_rect(n, n, CORNERS)
    pts = pts.copy()
    pts[:, 2] = 0.1 * np.sin(2 * pts[:, 0]) * np.cos(pts[:, 1])
    pts[:, :2] += 2.0
    args = (4, 4, 3, 2, 3, 2.5, "elasticRH3", "elasticRH3", [1.0, 0.25], pts, tris, float_type)
    op = RegularizedSparseIntegralOp(*args, farfield_op_type=FMMFarfieldOp(2.5, 8, 8, "fmm"))
    v = np.random.default_rng(6).random(tris.shape[0] * 9).astype(float_type)
    x = torch.from_numpy(v).cuda()
    seq = torch.empty(op.shape[0], dtype=x.dtype, device="cuda")
    assert not op._overlap_near()
    op.dot_device(x, seq)
    monkeypatch.setattr(RegularizedSparseIntegralOp, "OVERLAP_MIN_ROWS", 0)
    assert op._overlap_near()
    ov = torch.empty_like(seq)
    op.dot_device(x, ov)
    torch.cuda.synchronize()
    assert torch.equal(ov, seq)
    X = torch.stack([x, 2 * x])
    Y = torch.empty((2, op.shape[0]), dtype=x.dtype, device="cuda")
    op.dot_panel_device(X, Y)
    torch.cuda.synchronize()
    assert torch.equal(Y[0], seq)
    g, gx, gy = op.capture_graph()
    gx.copy_(x)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(gy, seq)
