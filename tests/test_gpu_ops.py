"""GPU parity of the drop-in operators (RegularizedSparseIntegralOp and
friends) against the oracle composition of the same operator."""
import numpy as np
import pytest

import tectosaur_b200 as tct
from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp

from helpers import PARAMS, bumpy_mesh, c1_mesh, oracle_sparse_op_dot, rel, two_surfaces

pytestmark = pytest.mark.gpu


def test_config1_matvec_fp64(cuda, orc):
    # Config 1: make_rect(20, 20) planar fault, 722 tris / 6498 DOF,
    # RegularizedSparseIntegralOp(6,6,6,2,5,2.5,'elasticRH3','elasticRH3',[1,.25]),
    # FP64, one matvec on x ~ N(0,1) seed 0.  Bar: 1e-10 relative.
    pts, tris = c1_mesh()
    assert tris.shape[0] == 722
    op = tct.RegularizedSparseIntegralOp(6, 6, 6, 2, 5, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, np.float64, TriToTriDirectFarfieldOp)
    assert op.shape == (6498, 6498)
    x = np.random.default_rng(0).standard_normal(op.shape[1])
    y = op.dot(x)
    want = oracle_sparse_op_dot(orc, 6, 6, 6, 2, 5, 2.5, "elasticRH3", "elasticRH3", PARAMS, pts,
                                tris, np.float64, x)
    assert rel(y, want) < 1e-10, rel(y, want)
    # no-correction apply = uncorrected nearfield blocks
    nc = op.nearfield_no_correction_dot(x)
    want_nc = oracle_sparse_op_dot(orc, 6, 6, 6, 2, 5, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                   pts, tris, np.float64, x, correction=False)
    far = op.farfield.dot(x)
    assert rel(nc + far, want_nc) < 1e-10


def test_config1_matvec_fp32(cuda, orc):
    pts, tris = c1_mesh()
    op = tct.RegularizedSparseIntegralOp(6, 6, 6, 2, 5, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, np.float32, TriToTriDirectFarfieldOp)
    x = np.random.default_rng(0).standard_normal(op.shape[1])
    y = op.dot(x)
    assert y.dtype == np.float32
    want64 = oracle_sparse_op_dot(orc, 6, 6, 6, 2, 5, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                  pts, tris, np.float64, x)
    want32 = oracle_sparse_op_dot(orc, 6, 6, 6, 2, 5, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                  pts, tris, np.float32, x)
    # the FP32 reference itself sits ~1e-6 from FP64; the device FP32 path
    # must match the FP32 oracle to float rounding and FP64 to 1e-5
    assert rel(y, want32) < 2e-5, rel(y, want32)
    assert rel(y, want64) < 1e-5, rel(y, want64)


@pytest.mark.parametrize("Kn,Kf", [("elasticU3", "elasticU3"), ("elasticT3", "elasticT3"),
                                   ("elasticRT3", "elasticRT3"), ("elasticRA3", "elasticRA3"),
                                   ("elasticH3", "elasticH3"), ("elasticRH3", "elasticH3")])
def test_sparse_op_kernels_fp64(cuda, orc, Kn, Kf):
    pts, tris = bumpy_mesh(8, seed=3)
    op = tct.RegularizedSparseIntegralOp(4, 4, 3, 2, 3, 2.0, Kn, Kf, [1.3, 0.3], pts, tris,
                                         np.float64, TriToTriDirectFarfieldOp)
    x = np.random.default_rng(1).standard_normal(op.shape[1])
    want = oracle_sparse_op_dot(orc, 4, 4, 3, 2, 3, 2.0, Kn, Kf, [1.3, 0.3], pts, tris,
                                np.float64, x)
    assert rel(op.dot(x), want) < 1e-10


def test_subsets(cuda, orc):
    # tests/test_integral_op.py:29-80 (op on obs/src subsets == rows/cols of the full op)
    pts, tris = tct.make_rect(10, 10, [[-1, 0, 1], [-1, 0, -1], [1, 0, -1], [1, 0, 1]])
    n = tris.shape[0]
    obs = np.arange(n // 2)
    src = np.arange(n // 4, n)
    args = (4, 4, 3, 2, 3, 2.0, "elasticRH3", "elasticRH3", PARAMS, pts, tris, np.float64,
            TriToTriDirectFarfieldOp)
    sub = tct.RegularizedSparseIntegralOp(*args, obs_subset=obs, src_subset=src)
    full = tct.RegularizedSparseIntegralOp(*args)
    x = np.random.default_rng(2).standard_normal(src.shape[0] * 9)
    xf = np.zeros(n * 9)
    xf[src[0] * 9:(src[-1] + 1) * 9] = x
    ys = sub.dot(x)
    yf = full.dot(xf)[:obs.shape[0] * 9]
    # The near-pair set of a subset operator comes from octrees built on the
    # subsets; the reference's leaf test reads radii by octree position, so a
    # few pairs within rounding of the threshold switch between near and far
    # (a far-rule vs accurate-rule difference, ~1e-6), as in the reference.
    assert rel(ys, yf) < 1e-4
    want = oracle_sparse_op_dot(orc, 4, 4, 3, 2, 3, 2.0, "elasticRH3", "elasticRH3", PARAMS, pts,
                                tris, np.float64, x, obs_subset=obs, src_subset=src)
    assert rel(ys, want) < 1e-10


def test_dense_equals_sparse(cuda):
    # RegularizedDenseIntegralOp (uncorrected near blocks + far blocks) and
    # RegularizedSparseIntegralOp (far everywhere + corrected near) are the
    # same matrix
    pts, tris = bumpy_mesh(6, seed=8)
    args = (4, 4, 3, 2, 3, 2.0, "elasticRH3", "elasticRH3", PARAMS, pts, tris, np.float64)
    dense = tct.RegularizedDenseIntegralOp(*args)
    sparse = tct.RegularizedSparseIntegralOp(*args, TriToTriDirectFarfieldOp)
    x = np.random.default_rng(4).standard_normal(sparse.shape[1])
    assert rel(dense.dot(x), sparse.dot(x)) < 1e-11


def test_nearfield_host_views(cuda):
    pts, tris = bumpy_mesh(5, seed=1)
    op = tct.RegularizedSparseIntegralOp(3, 3, 3, 2, 3, 2.0, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, np.float64, TriToTriDirectFarfieldOp)
    x = np.random.default_rng(0).standard_normal(op.shape[1])
    near = op.nearfield
    assert len(near.mat) == 4
    assert rel(np.asarray(near.full_scipy_mat().dot(x)).ravel(), near.dot(x)) < 1e-13
    assert rel(np.asarray(near.to_dense() @ x).ravel(), near.dot(x)) < 1e-13
    assert rel(sum(m.dot(x) for m in near.mat_no_correction), near.nearfield_no_correction_dot(x)) < 1e-13


def test_device_tensors_and_graph(cuda):
    torch = cuda
    pts, tris = bumpy_mesh(12, seed=6)
    op = tct.RegularizedSparseIntegralOp(3, 3, 3, 1, 3, 2.5, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, np.float32, TriToTriDirectFarfieldOp)
    x = np.random.default_rng(3).standard_normal(op.shape[1]).astype(np.float32)
    y_host = op.dot(x)
    xt = torch.from_numpy(x).cuda()
    y_dev = op.dot(xt)
    assert y_dev.is_cuda and np.array_equal(y_dev.cpu().numpy(), y_host)
    g, gx, gy = op.capture_graph()
    gx.copy_(xt)
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(gy.cpu().numpy(), y_host)
    # linearity of the apply
    x2 = np.random.default_rng(4).standard_normal(op.shape[1]).astype(np.float32)
    lhs = op.dot(2 * x - 3 * x2)
    rhs = 2 * y_host - 3 * op.dot(x2)
    assert rel(lhs, rhs) < 1e-5


def test_combinators(cuda):
    # tests/test_op_combinators.py and the T-problem operator of
    # examples/okada.py:354-358 (SumOp of H and a scaled MassOp)
    pts, tris = bumpy_mesh(5, seed=2)
    H = tct.RegularizedSparseIntegralOp(3, 3, 3, 2, 3, 2.0, "elasticRT3", "elasticRT3", PARAMS,
                                        pts, tris, np.float64, TriToTriDirectFarfieldOp)
    M = tct.MassOp(3, pts, tris)
    op = tct.SumOp([H, tct.MultOp(M, 0.5)])
    x = np.random.default_rng(0).standard_normal(H.shape[1])
    assert rel(op.dot(x), H.dot(x) + 0.5 * M.dot(x)) < 1e-14
    neg = tct.NegOp(H)
    assert rel(neg.dot(x), -H.dot(x)) == 0
    comp = tct.CompositeOp((H, 0, 0), (M, 0, H.shape[1]))
    xx = np.concatenate([x, x])
    assert rel(comp.dot(xx), H.dot(x) + M.dot(x)) < 1e-14


@pytest.mark.parametrize("td", [3, 1])
def test_mass_op_device_apply_matches_reference_matrix(cuda, golden, td):
    # ops/mass_op.py:9-42 + _mass_op.cpp:11-40: the reference's matrix (golden)
    # applied by the device block-diagonal BSR (tensor_dim 3) or CSR (1)
    g = golden("mass_op.npz")
    M = tct.MassOp(3, g["pts"], g["tris"], tensor_dim=td)
    A = g["mat_3_%d" % td]
    x = np.random.default_rng(1).standard_normal(A.shape[1])
    y = M.dot(x)
    assert y.dtype == np.float64
    assert rel(y, A @ x) < 1e-14
    xd = cuda.from_numpy(x.astype(np.float32)).cuda()
    yd = M.dot(xd)
    assert yd.is_cuda and yd.dtype == cuda.float32
    assert rel(yd.cpu().numpy(), A @ x) < 1e-6


def test_sum_with_mass_stays_on_device(cuda):
    # SumOp([H, MultOp(M, 0.5)]) (examples/okada.py:354-358) applied to a
    # device tensor: one device apply, no host round trip, in H's precision
    pts, tris = bumpy_mesh(6, seed=3)
    H = tct.RegularizedSparseIntegralOp(3, 3, 3, 2, 3, 2.0, "elasticRH3", "elasticRH3", PARAMS,
                                        pts, tris, np.float32, TriToTriDirectFarfieldOp)
    M = tct.MassOp(3, pts, tris)
    op = tct.SumOp([H, tct.MultOp(M, 0.5)])
    assert op.on_device()
    x = np.random.default_rng(0).standard_normal(H.shape[1]).astype(np.float32)
    yd = op.dot(cuda.from_numpy(x).cuda())
    assert yd.is_cuda and yd.dtype == cuda.float32
    want = H.dot(x).astype(np.float64) + 0.5 * (M.mat @ x.astype(np.float64))
    assert rel(yd.cpu().numpy(), want) < 1e-6
    y2 = cuda.ones_like(yd)
    op.dot_device(cuda.from_numpy(x).cuda(), y2, accumulate=True)
    assert rel(y2.cpu().numpy(), want + 1.0) < 1e-6
    neg = tct.NegOp(op)
    assert rel(neg.dot(x), -want) < 1e-6


def test_empty_nearfield_classes(cuda, orc):
    # two far-apart surfaces: no near, edge or vertex pairs across, only
    # coincident + in-surface classes; obs/src disjoint -> no coincident
    (pts, tris), s1, s2 = two_surfaces(n=5, sep=30.0)
    op = tct.RegularizedSparseIntegralOp(3, 3, 3, 2, 3, 2.0, "elasticRH3", "elasticRH3", PARAMS,
                                         pts, tris, np.float64, TriToTriDirectFarfieldOp,
                                         obs_subset=s1, src_subset=s2)
    assert op.nearfield.bsr.nnzb == 0
    x = np.random.default_rng(0).standard_normal(op.shape[1])
    from tectosaur_b200.util.quadrature import gauss2d_tri
    want = orc.farfield_tris("elasticRH3", np.float64, gauss2d_tri(2), pts, tris[s1], tris[s2], x,
                             PARAMS)
    assert rel(op.dot(x), want) < 1e-12


def test_reference_two_tri_vertex_adjacent(cuda, orc):
    # tests/test_integral_op.py:96-103 inputs (elasticH3, vertex-adjacent, nq 3)
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, -1, 0], [2, 0, 0]]).astype(np.float32)
    tris = np.array([[1, 2, 0], [1, 3, 4]]).astype(np.int32)
    from tectosaur_b200.nearfield.pairs_integrator import PairsIntegrator
    from tectosaur_b200.nearfield import triangle_rules as tr
    pi = PairsIntegrator("elasticH3", PARAMS, np.float32, 1, 1, pts, tris)
    out = pi.vert_adj(3, np.array([[0, 1, 0, 0]]))
    want = orc.pairs("elasticH3", np.float32, tr.vertex_adj_quad(3, 3, 3), pts, tris,
                     np.array([[0, 1, 0, 0, 0]]), PARAMS, adj=True, check0=True)
    assert rel(out, want) < 2e-5
