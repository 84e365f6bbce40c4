"""The allocation-free farfield entry point, through the C ABI.

tct_farfield_tris_matvec_noalloc exists for callers that cannot allocate
device memory when they apply the operator (inside a stream capture that
must not add memory nodes, under an application's own memory pool, or where
cudaMalloc's implicit synchronisation is unacceptable).  It takes only inputs
and outputs and runs on a fixed scratch array inside the library.  This file
checks, twice in a row (the scratch keeps the previous call's contents; the
second call is a smaller problem, so it lands on a scratch layout the first
call left different), that it returns what the workspace-taking entry point
returns for the same inputs, and that a problem larger than the built-in
scratch is refused with a message before any CUDA call (a CPU test: the
device pointers are NULL, so a refusal that stopped working would end at the
null-pointer check, never in a launch).  It runs last so that a failure here
leaves every other test already run; it passes alone in a fresh process as
well.
"""

import numpy as np
import pytest

from tectosaur_b200 import _lib
from tectosaur_b200.util import device
from tectosaur_b200.util.quadrature import gauss2d_tri

from helpers import PARAMS, bumpy_mesh, rel

TOL = {np.float32: 2e-5, np.float64: 1e-10}


def _inputs(ft, nq, seed, grid):
    pts, tris = bumpy_mesh(grid, seed=seed)
    obs = tris[::2]
    src = tris
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(src.shape[0] * 9)
    q = gauss2d_tri(nq)
    return (device.to_dev(pts, ft), device.to_dev(obs, np.int32), device.to_dev(src, np.int32),
            device.to_dev(x, ft), obs.shape[0], src.shape[0],
            np.ascontiguousarray(q[0], np.float64), np.ascontiguousarray(q[1], np.float64))


def _with_workspace(kid, prec, out, x, pts, obs, n_obs, src, n_src, qx, qw, params):
    nbytes = _lib.lib.tct_farfield_workspace_bytes(kid, prec, n_obs, n_src, qx.shape[0])
    ws = device.workspace(nbytes)
    _lib.check(_lib.lib.tct_farfield_tris_matvec(
        kid, prec, _lib.tptr(out), _lib.tptr(x), _lib.tptr(pts), _lib.tptr(obs), n_obs,
        _lib.tptr(src), n_src, qx.shape[0], _lib.dptr(qx), _lib.dptr(qw), _lib.dptr(params), 0,
        _lib.tptr(ws), nbytes, _lib.stream_ptr()), "tct_farfield_tris_matvec")


def _no_alloc(kid, prec, out, x, pts, obs, n_obs, src, n_src, qx, qw, params):
    _lib.check(_lib.lib.tct_farfield_tris_matvec_noalloc(
        kid, prec, _lib.tptr(out), _lib.tptr(x), _lib.tptr(pts), _lib.tptr(obs), n_obs,
        _lib.tptr(src), n_src, qx.shape[0], _lib.dptr(qx), _lib.dptr(qw), _lib.dptr(params), 0,
        _lib.stream_ptr()), "tct_farfield_tris_matvec_noalloc")


@pytest.mark.gpu
@pytest.mark.parametrize("K,ft,nq", [("elasticRH3", np.float32, 1), ("elasticRH3", np.float32, 2),
                                     ("elasticU3", np.float64, 2), ("elasticH3", np.float32, 1)])
def test_no_alloc_matches_workspace_entry_point(cuda, K, ft, nq):
    torch = cuda
    kid = _lib.kernel_id(K)
    prec = _lib.prec_of(ft)
    params = np.ascontiguousarray(PARAMS, np.float64)
    # a larger problem, then a smaller one: the second call's records and
    # partial sums sit on scratch bytes the first call wrote differently
    for call, grid in enumerate((40, 17)):
        pts, obs, src, x, n_obs, n_src, qx, qw = _inputs(ft, nq, seed=10 + call, grid=grid)
        want = device.zeros(n_obs * 9, ft)
        got = device.zeros(n_obs * 9, ft)
        _with_workspace(kid, prec, want, x, pts, obs, n_obs, src, n_src, qx, qw, params)
        _no_alloc(kid, prec, got, x, pts, obs, n_obs, src, n_src, qx, qw, params)
        torch.cuda.synchronize()
        w = want.cpu().numpy()
        g = got.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert rel(g, w) <= TOL[ft], (K, call, rel(g, w))


def test_no_alloc_rejects_oversized_problem():
    cap = _lib.lib.tct_farfield_noalloc_capacity()
    assert cap == 32 * 1024 * 1024
    n = 400_000  # needs more scratch than the built-in array holds
    params = np.ascontiguousarray(PARAMS, np.float64)
    q = gauss2d_tri(1)
    qx = np.ascontiguousarray(q[0], np.float64)
    qw = np.ascontiguousarray(q[1], np.float64)
    need = _lib.lib.tct_farfield_workspace_bytes(6, 0, n, n, 3)
    assert need > cap
    rc = _lib.lib.tct_farfield_tris_matvec_noalloc(
        6, 0, None, None, None, None, n, None, n, 3, _lib.dptr(qx), _lib.dptr(qw),
        _lib.dptr(params), 0, None)
    assert rc == _lib.TCT_ERR_ARG
    assert "scratch" in _lib.last_error()
    # negative sizes are refused as such, before the scratch size is asked
    rc = _lib.lib.tct_farfield_tris_matvec_noalloc(
        6, 0, None, None, None, None, -1, None, n, 3, _lib.dptr(qx), _lib.dptr(qw),
        _lib.dptr(params), 0, None)
    assert rc == _lib.TCT_ERR_ARG
    assert "negative size" in _lib.last_error()
    # no observation triangles: nothing to do, whatever the source count
    rc = _lib.lib.tct_farfield_tris_matvec_noalloc(
        6, 0, None, None, None, None, 0, None, n, 3, _lib.dptr(qx), _lib.dptr(qw),
        _lib.dptr(params), 0, None)
    assert rc == _lib.TCT_OK
