"""Batched persistent pair quadrature (mixed classes, orders and parameter
sets in one launch) against the oracle."""
import numpy as np
import pytest

from tectosaur_b200.nearfield import triangle_rules as tr
from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
from tectosaur_b200.nearfield.pairs_integrator import PairsIntegrator
from tectosaur_b200.util.quadrature import gauss4d_tri

from helpers import ALL_KERNELS, bumpy_mesh, rel

pytestmark = pytest.mark.gpu

PSETS = np.array([[1.0, 0.25], [1.3, 0.35]])


def mixed_workload(seed=0, orders=(2, 3, 4, 5, 7)):
    """Pairs of all four classes from a bumpy mesh, each pair assigned one of
    several quadrature orders and one of two parameter sets."""
    pts, tris = bumpy_mesh(8, seed=seed)
    n = tris.shape[0]
    cl = nearfield_pairs(pts, tris, np.arange(n), np.arange(n), 2.0)
    rng = np.random.default_rng(seed)
    rules, rule_key = [], {}

    def rid(kind, nq):
        key = (kind, nq)
        if key not in rule_key:
            if kind == "co":
                q, adj, c0 = tr.coincident_quad(nq), False, True
            elif kind == "ea":
                q, adj, c0 = tr.edge_adj_quad(nq), True, True
            elif kind == "va":
                q, adj, c0 = tr.vertex_adj_quad(nq, nq, nq), True, True
            else:
                q, adj, c0 = gauss4d_tri(nq, nq), False, False
            rule_key[key] = len(rules)
            rules.append((q[0], q[1], adj, c0))
        return rule_key[key]

    recs, rids, psets = [], [], []
    for kind in ["co", "ea", "va", "near"]:
        r = cl[kind][0]
        take = r[rng.permutation(r.shape[0])[:40]]
        for row in take:
            nq = int(rng.choice(orders))
            rec = np.zeros(5, np.int64)
            rec[:min(5, row.shape[0])] = row[:5]
            recs.append(rec)
            rids.append(rid(kind, nq))
            psets.append(int(rng.integers(0, 2)))
    return pts, tris, np.array(recs), np.array(rids), rules, np.array(psets)


@pytest.mark.parametrize("K", ALL_KERNELS)
def test_batched_vs_oracle_fp64(cuda, orc, K):
    pts, tris, recs, rids, rules, psets = mixed_workload(seed=1)
    pi = PairsIntegrator(K, PSETS[0], np.float64, 2, 3, pts, tris)
    # small chunk so that big rules are split over several warp items
    got = pi.batched(recs, rids, rules, psets, PSETS, chunk=256, small=64)
    want = np.zeros_like(got)
    for i in range(recs.shape[0]):
        q0, q1, adj, c0 = rules[rids[i]]
        want[i] = orc.pairs(K, np.float64, (q0, q1), pts, tris,
                            recs[i:i + 1, :5 if adj else 2], PSETS[psets[i]], adj=adj,
                            check0=c0)[0]
    assert np.all(np.isfinite(got))
    assert rel(got, want) < 1e-10, rel(got, want)


@pytest.mark.parametrize("K", ["elasticU3", "elasticH3", "elasticRH3", "elasticRT3"])
def test_batched_vs_oracle_fp32(cuda, orc, K):
    pts, tris, recs, rids, rules, psets = mixed_workload(seed=2, orders=(2, 3, 4))
    pi = PairsIntegrator(K, PSETS[0], np.float32, 2, 3, pts, tris)
    got = pi.batched(recs, rids, rules, psets, PSETS)
    want = np.zeros(got.shape)
    for i in range(recs.shape[0]):
        q0, q1, adj, c0 = rules[rids[i]]
        want[i] = orc.pairs(K, np.float32, (q0, q1), pts, tris,
                            recs[i:i + 1, :5 if adj else 2], PSETS[psets[i]], adj=adj,
                            check0=c0)[0]
    assert rel(got, want) < 2e-5, rel(got, want)


def test_batched_matches_per_class_launches(cuda):
    pts, tris = bumpy_mesh(9, seed=3)
    n = tris.shape[0]
    cl = nearfield_pairs(pts, tris, np.arange(n), np.arange(n), 2.5)
    pi = PairsIntegrator("elasticRH3", PSETS[0], np.float64, 2, 4, pts, tris)
    per = [pi.coincident(5, cl["co"][0]), pi.edge_adj(5, cl["ea"][0]),
           pi.vert_adj(4, cl["va"][0]), pi.nearfield(cl["near"][0])]
    rules = [(*tr.coincident_quad(5), False, True), (*tr.edge_adj_quad(5), True, True),
             (*tr.vertex_adj_quad(4, 4, 4), True, True), (*gauss4d_tri(4, 4), False, False)]
    recs, rids = [], []
    for k, kind in enumerate(["co", "ea", "va", "near"]):
        r = cl[kind][0]
        rr = np.zeros((r.shape[0], 5), np.int64)
        rr[:, :min(5, r.shape[1])] = r[:, :5]
        recs.append(rr)
        rids.append(np.full(r.shape[0], k))
    got = pi.batched(np.concatenate(recs), np.concatenate(rids), rules)
    want = np.concatenate(per)
    assert rel(got, want) < 1e-12


def test_batched_c3_sample_vs_oracle_fp64(cuda, orc):
    """A sample of the benchmark's random pair workload (all four classes,
    orders 3..20, seven kernels, two nu values): every pair's 81 values
    against the oracle."""
    import bench
    P, T, recs, owner, attr = bench.c3_pairs(160, seed=21)
    groups = bench.c3_groups(recs, owner, attr)
    psets = np.array([[1.0, 0.25], [1.0, 0.35]])
    checked = 0
    for K, g in groups.items():
        pi = PairsIntegrator(K, psets[0], np.float64, 2, 2, P, T)
        got = pi.batched(g["recs"], g["rule_ids"], g["rules"], g["nu"], psets)
        for i in range(0, g["recs"].shape[0], 3):
            pts4, wts, adj, c0 = g["rules"][g["rule_ids"][i]]
            want = orc.pairs(K, np.float64, (pts4, wts), P, T,
                             g["recs"][i:i + 1, :5 if adj else 2], psets[g["nu"][i]], adj=adj,
                             check0=c0)[0]
            assert rel(got[i], want) < 1e-10, (K, i, rel(got[i], want))
            checked += 1
    assert checked > 40
