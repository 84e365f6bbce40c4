"""Corrected nearfield operator (reference: tectosaur/nearfield/nearfield_op.py:24-168).

Construction follows the reference step for step:
  * coincident pairs = obs_subset ∩ src_subset, integrated with the
    Erichsen–Sauter rule (r^2 == 0 points skipped);
  * close-or-touching pairs from the near-pair search, split into
    edge-adjacent (oriented by resolve_ea_rotation), vertex-adjacent and
    separate-but-near pairs, integrated with the Sauter–Schwab edge rule, the
    polar vertex rule and a gauss4d_tri(nq_near) product rule;
  * from every class the same pairs integrated with the farfield rule
    gauss4d_tri(nq_far) and the farfield kernel are subtracted, because the
    farfield operator is applied to all pairs (nearfield_op.py:94-141).

B200 layout: all four classes share one device BSR matrix whose blocks the
pair kernels write in place (accurate rule, then the correction subtracted
into the same slots), so the nearfield apply is a single tct_bsr9_matvec.
The build integrates every class in one persistent launch of the batched
pair kernel (work queues of uneven rules: the reference launches one
single_pairs kernel per class and rule, nearfield/pairs_integrator.py:43-68)
and all the corrections in a second; ``batched=False`` keeps the per-class
launches.
The uncorrected blocks (``nearfield_no_correction_dot``) are kept as the
correction array C beside the corrected array D (no-correction = D + C);
``keep_uncorrected=False`` drops C to halve the footprint.

Block order: canonical, by (obs dof row, src dof column); the reference
orders a row's blocks by thread-completion order of its near-pair search,
which only changes the floating-point summation order of the apply.
"""
import numpy as np

from .. import _lib
from ..mesh import find_near_adj
from ..util import device
from ..util.sparse import BCOOMatrix, DeviceBSR9
from .pairs_integrator import PairsIntegrator


def to_dof_space(tri_indices, obs_subset, src_subset):
    """Map (obs tri, src tri) pairs to positions within the subsets
    (nearfield_op.py:24-38; first occurrence when a subset repeats)."""
    tri_indices = np.asarray(tri_indices).reshape(-1, 2)
    if tri_indices.shape[0] == 0:
        return np.empty((0, 2), dtype=np.int64)
    n = int(max(np.max(obs_subset), np.max(src_subset), np.max(tri_indices))) + 1
    opos = np.full(n, -1, dtype=np.int64)
    spos = np.full(n, -1, dtype=np.int64)
    opos[np.asarray(obs_subset)[::-1]] = np.arange(len(obs_subset))[::-1]
    spos[np.asarray(src_subset)[::-1]] = np.arange(len(src_subset))[::-1]
    out = np.stack([opos[tri_indices[:, 0]], spos[tri_indices[:, 1]]], axis=1)
    if np.any(out < 0):
        raise ValueError("pair references a triangle outside the obs/src subsets")
    return out


def to_tri_space(dof_indices, obs_subset, src_subset):
    dof_indices = np.asarray(dof_indices)
    tri_idxs = np.array([np.asarray(obs_subset)[dof_indices[:, 0]],
                         np.asarray(src_subset)[dof_indices[:, 1]]]).T
    return np.concatenate((tri_idxs.reshape(-1, 2), dof_indices[:, 2:]), axis=1)


def edge_adj_orient(touching_verts):
    tv = sorted(touching_verts)
    if tv[0] == 0:
        if tv[1] == 2:
            return 2
        return 0
    return 1


def resolve_ea_rotation(tris, ea):
    """(obs, src, obs_clicks, src_clicks, src_flip) for edge-adjacent rows
    (obs, src, obs corner a, src corner a, obs corner b, src corner b)
    (nearfield_op.py:52-62); computed in libtct_b200.so."""
    ea = np.ascontiguousarray(np.asarray(ea), dtype=np.int64).reshape(-1, 6)
    t = np.ascontiguousarray(tris, dtype=np.int64)
    out = np.empty((ea.shape[0], 5), dtype=np.int64)
    if ea.shape[0]:
        _lib.check(_lib.lib.tct_resolve_ea_rotation(_lib.i64ptr(t), _lib.i64ptr(ea), ea.shape[0],
                                                     _lib.i64ptr(out)), "tct_resolve_ea_rotation")
    return out


def restrict_rows(classes, row_range):
    """Keep the pairs whose dof row lies in [r0, r1) and renumber the rows
    from 0: the block rows r0..r1-1 of the operator the classes describe."""
    r0, r1 = row_range
    out = {}
    for c, (recs, dofs) in classes.items():
        m = (dofs[:, 0] >= r0) & (dofs[:, 0] < r1)
        d = dofs[m].copy()
        d[:, 0] -= r0
        out[c] = (recs[m], d)
    return out


def nearfield_pairs(pts, tris, obs_subset, src_subset, near_threshold, row_range=None):
    """Host-side pair classes: dict of tri-space records and dof-space
    (row, col) for 'co', 'ea', 'va', 'near' (nearfield_op.py:95-114).

    row_range=(r0, r1) (an addition, for row shards): the search still runs
    over the whole obs_subset, so the pair set is the full operator's, and
    only the pairs of dof rows r0..r1-1 are kept (rows renumbered from 0).
    Searching the shard's triangles alone would build different octrees, and
    the reference's leaf test reads radii by tree position, so pairs at the
    threshold could change."""
    obs_subset = np.asarray(obs_subset)
    src_subset = np.asarray(src_subset)
    co_tris = np.intersect1d(obs_subset, src_subset)
    co = np.array([co_tris, co_tris]).T.reshape(-1, 2).astype(np.int64)
    co_dofs = to_dof_space(co, obs_subset, src_subset)
    close = find_near_adj.find_close_or_touching(pts, tris[obs_subset], pts, tris[src_subset],
                                                 near_threshold)
    near_dofs, va_dofs, ea_dofs = find_near_adj.split_adjacent_close(
        close, tris[obs_subset], tris[src_subset])
    near = to_tri_space(near_dofs, obs_subset, src_subset)
    va = to_tri_space(va_dofs, obs_subset, src_subset)
    va = np.hstack((va, np.zeros((va.shape[0], 1), dtype=np.int64)))
    ea = resolve_ea_rotation(tris, to_tri_space(ea_dofs, obs_subset, src_subset))
    out = {
        "co": (co, co_dofs),
        "ea": (ea, ea_dofs[:, :2]),
        "va": (va, va_dofs[:, :2]),
        "near": (near, near_dofs),
    }
    return out if row_range is None else restrict_rows(out, row_range)


CLASSES = ("co", "ea", "va", "near")


class RegularizedNearfieldIntegralOp:
    def __init__(self, pts, tris, obs_subset, src_subset,
                 nq_coincident, nq_edge_adj, nq_vert_adjacent,
                 nq_far, nq_near, near_threshold,
                 K_near_name, K_far_name, params, float_type, keep_uncorrected=True,
                 row_range=None, batched=True):
        device.require_cuda()
        pts = np.asarray(pts, dtype=np.float64)
        tris = np.asarray(tris, dtype=np.int64)
        obs_subset = np.asarray(obs_subset)
        src_subset = np.asarray(src_subset)
        self.float_type = np.dtype(float_type)
        # row_range (an addition): this operator is block rows r0..r1-1 of the
        # one over obs_subset -- the same pairs and blocks (see nearfield_pairs)
        self.row_range = row_range
        n_rows = obs_subset.shape[0] if row_range is None else row_range[1] - row_range[0]
        self.shape = (n_rows * 9, src_subset.shape[0] * 9)

        pairs_int = PairsIntegrator(K_near_name, params, float_type, nq_far, nq_near, pts, tris)
        corr_int = PairsIntegrator(K_far_name, params, float_type, nq_far, nq_near, pts, tris)
        self.classes = nearfield_pairs(pts, tris, obs_subset, src_subset, near_threshold,
                                       row_range=row_range)

        rows = np.concatenate([self.classes[c][1][:, 0] for c in CLASSES]).astype(np.int64)
        cols = np.concatenate([self.classes[c][1][:, 1] for c in CLASSES]).astype(np.int64)
        order = np.lexsort((cols, rows))  # stable: duplicates keep class order
        slot = np.empty_like(order)
        slot[order] = np.arange(order.shape[0])
        n_row_blocks = n_rows
        indptr = np.zeros(n_row_blocks + 1, dtype=np.int64)
        np.add.at(indptr, rows + 1, 1)
        indptr = np.cumsum(indptr)
        self.bsr = DeviceBSR9(self.shape, indptr, cols[order], float_type, row_align="auto")
        self.class_slots = {}  # CSR positions of each class's blocks
        start = 0
        for c in CLASSES:
            n = self.classes[c][1].shape[0]
            self.class_slots[c] = slot[start:start + n]
            start += n
        self.correction = device.zeros(81 * self.bsr.stride, float_type) \
            if keep_uncorrected else None

        stride = self.bsr.stride
        self.n_pairs = {c: self.classes[c][1].shape[0] for c in CLASSES}
        if batched:
            self._integrate_batched(pairs_int, corr_int, nq_coincident, nq_edge_adj,
                                    nq_vert_adjacent, nq_far, nq_near, stride)
            self._mats = None
            return
        rules = {
            "co": (pairs_int.coincident_rule(nq_coincident), False, True),
            "ea": (pairs_int.edge_adj_rule(nq_edge_adj), True, True),
            "va": (pairs_int.vert_adj_rule(nq_vert_adjacent), True, True),
            "near": (pairs_int.near_rule(), False, False),
        }
        far_rule = corr_int.far_rule()
        for c in CLASSES:
            recs, dofs = self.classes[c]
            n = dofs.shape[0]
            if n == 0:
                continue
            rule, adj, check0 = rules[c]
            rec_dev = device.to_dev(np.ascontiguousarray(recs[:, :5 if adj else 2]), np.int32)
            slot_dev = device.to_dev(self.bsr.slots(self.class_slots[c]), np.int32)
            pairs_int.integrate_into(self.bsr.data, rule, rec_dev, n, adj, check0,
                                     slot=slot_dev, slot_stride=stride)
            base_dev = rec_dev if not adj else device.to_dev(
                np.ascontiguousarray(recs[:, :2]), np.int32)
            corr_check0 = c == "co"
            corr_int.integrate_into(self.bsr.data, far_rule, base_dev, n, False, corr_check0,
                                    slot=slot_dev, slot_stride=stride, sign=-1, accumulate=True)
            if self.correction is not None:
                corr_int.integrate_into(self.correction, far_rule, base_dev, n, False,
                                        corr_check0, slot=slot_dev, slot_stride=stride)
        self._mats = None

    def _integrate_batched(self, pairs_int, corr_int, nq_co, nq_ea, nq_va, nq_far, nq_near,
                           stride):
        """All four classes in one persistent launch of the batched pair
        kernel (tct_pairs_integrate_batched_slots: the coincident, edge- and
        vertex-adjacent rules as warp items, the near rule as thread items),
        written into the BSR slots; then the far-rule corrections of every
        pair in one launch, subtracted in place (and written to the
        uncorrected-form array C when kept).  No pair is split, so the
        blocks do not depend on the launch's scheduling."""
        from ..util.quadrature import gauss4d_tri
        from . import triangle_rules
        host_rules = {
            "co": (triangle_rules.coincident_quad(nq_co), False, True),
            "ea": (triangle_rules.edge_adj_quad(nq_ea), True, True),
            "va": (triangle_rules.vertex_adj_quad(nq_va, nq_va, nq_va), True, True),
            "near": (gauss4d_tri(nq_near, nq_near), False, False),
        }
        far_q = gauss4d_tri(nq_far, nq_far)
        groups, corr_groups, slots = [], [], []
        for c in CLASSES:
            recs, dofs = self.classes[c]
            n = dofs.shape[0]
            if n == 0:
                continue
            (qp, qw), adj, check0 = host_rules[c]
            base = np.zeros((n, 5), dtype=np.int64)
            base[:, :2] = recs[:, :2]
            r5 = recs[:, :5] if adj else base
            groups.append((r5, (qp, qw, adj, check0)))
            corr_groups.append((base, (far_q[0], far_q[1], False, c == "co")))
            slots.append(self.bsr.slots(self.class_slots[c]))
        if not groups:
            return
        slot_dev = device.to_dev(np.concatenate(slots).astype(np.int32))
        plan = pairs_int.class_plan(groups)
        pairs_int.batched_run_slots(plan, self.bsr.data, slot_dev, stride, 1.0, add=False)
        del plan
        cplan = corr_int.class_plan(corr_groups)
        corr_int.batched_run_slots(cplan, self.bsr.data, slot_dev, stride, -1.0, add=True)
        if self.correction is not None:
            corr_int.batched_run_slots(cplan, self.correction, slot_dev, stride, 1.0, add=False)

    # -- apply ------------------------------------------------------------
    def dot_device(self, x, y, accumulate=False, stream=None):
        """y (+)= Near x on device tensors of float_type."""
        return self.bsr.matvec(x, y, accumulate=accumulate, stream=stream)

    def dot_panel_device(self, X, Y, accumulate=False, stream=None):
        """Y[r] (+)= Near X[r] for device tensors X (R, n_cols), Y (R, n_rows)."""
        return self.bsr.matvec_panel(X, Y, accumulate=accumulate, stream=stream)

    def _host_or_device(self, v, fn):
        if device.is_device_tensor(v):
            x = v.to(device.torch_dtype(self.float_type)).contiguous()
            y = device.empty(self.shape[0], self.float_type)
            fn(x, y)
            return y
        x = device.to_dev(np.asarray(v).reshape(-1), self.float_type)
        y = device.empty(self.shape[0], self.float_type)
        fn(x, y)
        return y.cpu().numpy()

    def dot(self, v):
        return self._host_or_device(v, lambda x, y: self.bsr.matvec(x, y))

    def nearfield_no_correction_dot(self, v):
        if self.correction is None:
            raise RuntimeError("built with keep_uncorrected=False")
        return self._host_or_device(
            v, lambda x, y: self.bsr.matvec(x, y, extra=self.correction))

    def astype(self, float_type, keep_uncorrected=True):
        """The same nearfield in another precision: the block structure is
        shared and the blocks are cast (not re-integrated)."""
        import copy
        twin = copy.copy(self)
        twin.float_type = np.dtype(float_type)
        tdt = device.torch_dtype(float_type)
        twin.bsr = copy.copy(self.bsr)
        twin.bsr.float_type = twin.float_type
        twin.bsr.data = self.bsr.data.to(tdt)
        twin.correction = (self.correction.to(tdt)
                           if keep_uncorrected and self.correction is not None else None)
        twin._mats = None
        return twin

    # -- host views (reference attributes) --------------------------------
    def _build_mats(self):
        D = self.bsr.blocks_host()
        C = self.bsr.blocks_host(self.correction) if self.correction is not None else None
        mats, mats_nc = [], []
        for c in CLASSES:
            dofs = self.classes[c][1]
            s = self.class_slots[c]
            mats.append(BCOOMatrix(dofs[:, 0].copy(), dofs[:, 1].copy(), D[s], self.shape))
            if C is not None:
                mats_nc.append(BCOOMatrix(dofs[:, 0].copy(), dofs[:, 1].copy(), D[s] + C[s],
                                          self.shape))
        self._mats = (mats, mats_nc)

    @property
    def mat(self):
        if self._mats is None:
            self._build_mats()
        return self._mats[0]

    @property
    def mat_no_correction(self):
        if self._mats is None:
            self._build_mats()
        return self._mats[1]

    def full_scipy_mat(self):
        return sum([m.to_bsr().to_scipy() for m in self.mat])

    def full_scipy_mat_no_correction(self):
        return sum([m.to_bsr().to_scipy() for m in self.mat_no_correction])

    def to_dense(self):
        return sum([m.to_bsr().to_scipy().todense() for m in self.mat])

    def no_correction_to_dense(self):
        return sum([m.to_bsr().to_scipy().todense() for m in self.mat_no_correction])
