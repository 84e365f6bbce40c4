"""Multi-RHS point farfield on the tensor cores (tct_farfield_pts_panel,
csrc/pts_mrhs.cu) against the single-vector point kernel applied vector by
vector and against the FP64 oracle (farfield_direct.cl:15-113 restated)."""
import numpy as np
import pytest

from tectosaur_b200.farfield import farfield_pts_direct, farfield_pts_panel

from helpers import PARAMS, rel

pytestmark = pytest.mark.gpu


def _cloud(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-scale, scale, (n, 3))
    nrm = rng.standard_normal((n, 3))
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    return p, nrm


@pytest.mark.parametrize("K", ["elasticU3", "elasticT3", "elasticA3", "elasticH3"])
@pytest.mark.parametrize("n_obs,n_src,R", [(300, 500, 20), (1000, 2003, 16), (129, 7, 3)])
def test_pts_panel_matches_per_vector(cuda, K, n_obs, n_src, R):
    op, on = _cloud(n_obs, 1)
    sp, sn = _cloud(n_src, 2)
    V = np.random.default_rng(3).standard_normal((R, 3 * n_src)).astype(np.float32)
    got = farfield_pts_panel(K, op, on, sp, sn, V, PARAMS)
    assert got.shape == (R, 3 * n_obs) and np.all(np.isfinite(got))
    for r in range(R):
        want = farfield_pts_direct(K, op, on, sp, sn, V[r], PARAMS, np.float32)
        assert rel(got[r], want) < 2e-5, (K, r, rel(got[r], want))


@pytest.mark.parametrize("K", ["elasticT3", "elasticH3"])
def test_pts_panel_vs_fp64_oracle_with_coincident_points(cuda, orc, K):
    # the source points include every observation point: r^2 == 0 pairs skip
    sp, sn = _cloud(3000, 4, scale=3.0)
    op, on = sp[::3].copy(), sn[::3].copy()
    V = np.random.default_rng(5).standard_normal((16, 3 * sp.shape[0])).astype(np.float32)
    got = farfield_pts_panel(K, op, on, sp, sn, V, PARAMS)
    for r in (0, 7, 15):
        want = orc.farfield_pts(K, np.float64, op, on, sp, sn, V[r].astype(np.float64), PARAMS)
        assert rel(got[r], want) < 1e-5, (K, r, rel(got[r], want))
