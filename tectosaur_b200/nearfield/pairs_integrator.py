"""Triangle-pair quadrature on the device (reference:
tectosaur/nearfield/pairs_integrator.py:27-93, kernels single_pairs{Z,N}[_adj]
of tectosaur/assemble.cl:24-103).

Same constructor and methods as the reference's PairsIntegrator; each method
returns the (n, 3, 3, 3, 3) blocks as a host array in float_type.  The
nearfield operator uses ``integrate_into`` instead, which writes the blocks
straight into the device BSR matrix (no host round trip, no 2^17-pair
chunking: one launch per pair class).
"""
import numpy as np

from .. import _lib
from ..kernels import kernels
from ..util import device
from ..util.quadrature import gauss4d_tri
from . import triangle_rules


class PairsIntegrator:
    def __init__(self, kernel, params, float_type, nq_far, nq_near, pts, tris):
        if kernel not in kernels:
            raise ValueError("unknown kernel %r" % kernel)
        self.kernel = kernel
        self.kid = _lib.kernel_id(kernel)
        self.params = np.ascontiguousarray(np.asarray(params, dtype=np.float64)[:2])
        self.float_type = np.dtype(float_type)
        self.prec = _lib.prec_of(float_type)
        self.nq_far = nq_far
        self.nq_near = nq_near
        self.gpu_pts = device.to_dev(np.asarray(pts, dtype=np.float64), self.float_type)
        self.gpu_tris = device.to_dev(np.asarray(tris), np.int32)
        self._rules = {}

    def _rule(self, key, make):
        if key not in self._rules:
            q = make()
            self._rules[key] = (device.to_dev(q[0], self.float_type),
                                device.to_dev(q[1], self.float_type), q[0].shape[0])
        return self._rules[key]

    def far_rule(self):
        return self._rule(("far", self.nq_far), lambda: gauss4d_tri(self.nq_far, self.nq_far))

    def near_rule(self):
        return self._rule(("near", self.nq_near), lambda: gauss4d_tri(self.nq_near, self.nq_near))

    def coincident_rule(self, nq):
        return self._rule(("co", nq), lambda: triangle_rules.coincident_quad(nq))

    def edge_adj_rule(self, nq):
        return self._rule(("ea", nq), lambda: triangle_rules.edge_adj_quad(nq))

    def vert_adj_rule(self, nq):
        if isinstance(nq, (int, np.integer)):
            nq = (nq, nq, nq)
        nq = tuple(int(v) for v in nq)
        return self._rule(("va",) + nq, lambda: triangle_rules.vertex_adj_quad(*nq))

    def integrate_into(self, out, rule, pairs_dev, n_pairs, adj, check0, slot=None,
                       slot_stride=0, sign=1, accumulate=False, stream=None):
        """Launch one pair class: blocks of `pairs_dev` (int32 records of 2 or
        5 ints) under `rule`, written (or added, times `sign`) to `out`."""
        if n_pairs == 0:
            return
        qp, qw, nq = rule
        _lib.check(_lib.lib.tct_pairs_integrate(
            self.kid, self.prec, int(adj), int(check0), _lib.tptr(out),
            _lib.tptr(slot) if slot is not None else None, int(slot_stride), int(sign),
            int(bool(accumulate)), nq, _lib.tptr(qp), _lib.tptr(qw), _lib.tptr(self.gpu_pts),
            _lib.tptr(self.gpu_tris), _lib.tptr(pairs_dev), int(n_pairs),
            _lib.dptr(self.params), _lib.stream_ptr(stream)), "tct_pairs_integrate")

    def pairs_quad(self, rule, pairs_list, adj, check0):
        pairs_list = np.asarray(pairs_list)
        n = pairs_list.shape[0]
        if n == 0:
            return np.empty((0, 3, 3, 3, 3), dtype=self.float_type)
        rec = pairs_list.reshape(n, -1)[:, :5 if adj else 2].astype(np.int32)
        if adj and rec.shape[1] < 5:
            # a 4-column vertex-adjacent record has no flip column: flip = 0
            rec = np.hstack((rec, np.zeros((n, 5 - rec.shape[1]), dtype=np.int32)))
        rec = np.ascontiguousarray(rec)
        out = device.empty(n * 81, self.float_type)
        self.integrate_into(out, rule, device.to_dev(rec), n, adj, check0)
        return out.cpu().numpy().reshape((n, 3, 3, 3, 3))

    def batched_plan(self, records, rule_ids, rules, param_set_ids=None, param_sets=None,
                     chunk=4096, small=768):
        """Work plan of one batched launch, uploaded to the device once.

        records: (n, 5) int (obs, src, obs_clicks, src_clicks, src_flip);
        rule_ids: (n,) index into `rules`, a list of (pts (m, 4), wts (m,),
        adjacent, check0); param_set_ids: (n,) index into `param_sets`
        ((k, 2) [mu, nu], k <= 8; default: this integrator's params).
        Work schedule: pairs whose rule has <= `small` points are whole-pair
        thread items; larger ones are cut into warp items of <= `chunk`
        points; each queue is ordered by decreasing size."""
        records = np.asarray(records).reshape(-1, 5).astype(np.int64)
        n = records.shape[0]
        rule_ids = np.asarray(rule_ids, dtype=np.int64).reshape(n)
        if param_sets is None:
            param_sets = self.params.reshape(1, 2)
        param_sets = np.ascontiguousarray(np.asarray(param_sets, dtype=np.float64).reshape(-1, 2))
        if param_set_ids is None:
            param_set_ids = np.zeros(n, dtype=np.int64)
        sizes = np.array([r[0].shape[0] for r in rules], dtype=np.int64)
        rule_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        rule_flags = np.array([(1 if r[2] else 0) | (2 if r[3] else 0) for r in rules], np.int32)
        pts_all = np.concatenate([np.asarray(r[0], np.float64).reshape(-1, 4) for r in rules])
        wts_all = np.concatenate([np.asarray(r[1], np.float64).reshape(-1) for r in rules])
        rec7 = np.concatenate([records, rule_ids[:, None], np.asarray(param_set_ids)[:, None]],
                              axis=1).astype(np.int32)
        psize = sizes[rule_ids]
        big = psize > small
        # warp items: split large pairs into chunks
        bp = np.nonzero(big)[0]
        nchunk = (psize[bp] + chunk - 1) // chunk
        wi_pair = np.repeat(bp, nchunk)
        first = np.concatenate([np.arange(k) for k in nchunk]) * chunk if bp.size else \
            np.zeros(0, np.int64)
        wi_p0 = first
        wi_p1 = np.minimum(first + chunk, psize[wi_pair])
        wi_split = np.repeat((nchunk > 1).astype(np.int64), nchunk)
        # largest items first (load balance); among equal sizes, grouped by
        # rule and rule segment, so that the warps running at the same time
        # read the same rule points (from L2, not HBM)
        order = np.lexsort((wi_p0, rule_ids[wi_pair], -(wi_p1 - wi_p0)))
        witems = np.stack([wi_pair, wi_p0, wi_p1, wi_split], axis=1)[order]
        tp = np.nonzero(~big)[0]
        tp = tp[np.lexsort((rule_ids[tp], -psize[tp]))]
        titems = np.stack([tp, np.zeros_like(tp), psize[tp], np.zeros_like(tp)], axis=1)
        items = np.ascontiguousarray(np.concatenate([witems, titems]).astype(np.int32))
        ft = self.float_type
        plan = dict(n=n, n_warp=witems.shape[0], n_thread=titems.shape[0],
                    param_sets=param_sets, n_points=int(psize.sum()),
                    ws=device.workspace(2048),
                    dev=[device.to_dev(rec7), device.to_dev(rule_off),
                         device.to_dev(rule_flags), device.to_dev(pts_all, ft),
                         device.to_dev(wts_all, ft),
                         device.to_dev(items if items.size else np.zeros((1, 4), np.int32))])
        return plan

    def class_plan(self, classes, small=768):
        """Work plan for groups of pairs that share a rule (the nearfield
        operator's classes), no pair split: classes = [(records (n, 5), rule
        (pts, wts, adjacent, check0))].  Pairs of rules above `small` points
        are warp items (the 32 lanes stride over the rule), the others thread
        items; both queues run the larger rules first and keep each class
        contiguous, so no sort of the (possibly 10^8) pairs is needed.
        Deterministic: every block is summed in a fixed order by one warp or
        one thread.  Pair p of the plan is the p-th record in class order."""
        groups = [(np.asarray(r).reshape(-1, 5), q) for r, q in classes]
        rules = [q for _, q in groups]
        sizes = np.array([q[0].shape[0] for q in rules], dtype=np.int64)
        rule_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        rule_flags = np.array([(1 if q[2] else 0) | (2 if q[3] else 0) for q in rules], np.int32)
        pts_all = np.concatenate([np.asarray(q[0], np.float64).reshape(-1, 4) for q in rules])
        wts_all = np.concatenate([np.asarray(q[1], np.float64).reshape(-1) for q in rules])
        n = int(sum(r.shape[0] for r, _ in groups))
        rec7 = np.empty((n, 7), dtype=np.int32)
        starts = np.concatenate([[0], np.cumsum([r.shape[0] for r, _ in groups])]).astype(np.int64)
        for g, (r, _) in enumerate(groups):
            rec7[starts[g]:starts[g + 1], :5] = r
            rec7[starts[g]:starts[g + 1], 5] = g
        rec7[:, 6] = 0
        witems, titems = [], []
        for g in np.argsort(-sizes, kind="stable"):
            k = np.arange(starts[g], starts[g + 1], dtype=np.int64)
            it = np.stack([k, np.zeros_like(k), np.full_like(k, sizes[g]), np.zeros_like(k)],
                          axis=1)
            (witems if sizes[g] > small else titems).append(it)
        witems = np.concatenate(witems) if witems else np.zeros((0, 4), np.int64)
        titems = np.concatenate(titems) if titems else np.zeros((0, 4), np.int64)
        items = np.ascontiguousarray(np.concatenate([witems, titems]).astype(np.int32))
        ft = self.float_type
        return dict(n=n, n_warp=witems.shape[0], n_thread=titems.shape[0],
                    param_sets=self.params.reshape(1, 2), n_points=int(sizes[rec7[:, 5]].sum()),
                    ws=device.workspace(2048),
                    dev=[device.to_dev(rec7), device.to_dev(rule_off),
                         device.to_dev(rule_flags), device.to_dev(pts_all, ft),
                         device.to_dev(wts_all, ft),
                         device.to_dev(items if items.size else np.zeros((1, 4), np.int32))])

    def batched_run_slots(self, plan, out, slot_dev, slot_stride, sign=1.0, add=False,
                          stream=None):
        """Launch a plan writing pair p's block into the structure-of-arrays
        array `out` at slot slot_dev[p] (element e at e * slot_stride + slot),
        times sign, added to the destination when `add`."""
        if plan["n"] == 0:
            return out
        d = plan["dev"]
        _lib.check(_lib.lib.tct_pairs_integrate_batched_slots(
            self.kid, self.prec, _lib.tptr(out), _lib.tptr(slot_dev), int(slot_stride),
            float(sign), int(bool(add)), plan["n"], _lib.tptr(self.gpu_pts),
            _lib.tptr(self.gpu_tris), _lib.tptr(d[0]), _lib.tptr(d[1]), _lib.tptr(d[2]),
            _lib.tptr(d[3]), _lib.tptr(d[4]), _lib.tptr(d[5]), plan["n_warp"],
            plan["n_thread"], _lib.dptr(plan["param_sets"]), plan["param_sets"].shape[0],
            _lib.tptr(plan["ws"]), 2048, _lib.stream_ptr(stream)),
            "tct_pairs_integrate_batched_slots")
        return out

    def batched_run(self, plan, out=None, stream=None):
        """Launch a batched plan: out (n * 81 device array, allocated when
        None) receives the blocks (before any correction)."""
        out = out if out is not None else device.empty(max(plan["n"] * 81, 1), self.float_type)
        d = plan["dev"]
        _lib.check(_lib.lib.tct_pairs_integrate_batched(
            self.kid, self.prec, _lib.tptr(out), plan["n"], _lib.tptr(self.gpu_pts),
            _lib.tptr(self.gpu_tris), _lib.tptr(d[0]), _lib.tptr(d[1]), _lib.tptr(d[2]),
            _lib.tptr(d[3]), _lib.tptr(d[4]), _lib.tptr(d[5]), plan["n_warp"],
            plan["n_thread"], _lib.dptr(plan["param_sets"]), plan["param_sets"].shape[0], 0,
            _lib.tptr(plan["ws"]), 2048, _lib.stream_ptr(stream)), "tct_pairs_integrate_batched")
        return out

    def batched_device(self, records, rule_ids, rules, param_set_ids=None, param_sets=None,
                       chunk=4096, small=768, out=None, stream=None):
        """All pairs of mixed classes and orders in one persistent launch
        (plan + run); returns the (n * 81) device array of blocks."""
        plan = self.batched_plan(records, rule_ids, rules, param_set_ids, param_sets, chunk,
                                 small)
        out = self.batched_run(plan, out, stream)
        self._batched_keepalive = plan
        return out

    def batched(self, records, rule_ids, rules, param_set_ids=None, param_sets=None, **kw):
        """Host (n, 3, 3, 3, 3) blocks of batched_device."""
        n = np.asarray(records).reshape(-1, 5).shape[0]
        if n == 0:
            return np.empty((0, 3, 3, 3, 3), dtype=self.float_type)
        out = self.batched_device(records, rule_ids, rules, param_set_ids, param_sets, **kw)
        return out[:n * 81].cpu().numpy().reshape(n, 3, 3, 3, 3)

    def correction(self, pairs_list, check0):
        return self.pairs_quad(self.far_rule(), pairs_list, False, check0)

    def nearfield(self, pairs_list):
        return self.pairs_quad(self.near_rule(), pairs_list, False, False)

    def vert_adj(self, nq, pairs_list):
        return self.pairs_quad(self.vert_adj_rule(nq), pairs_list, True, True)

    def coincident(self, nq, pairs_list):
        return self.pairs_quad(self.coincident_rule(nq), pairs_list, False, True)

    def edge_adj(self, nq, pairs_list):
        return self.pairs_quad(self.edge_adj_rule(nq), pairs_list, True, True)
