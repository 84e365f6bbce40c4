"""Block-composed operator (reference: tectosaur/ops/composite_op.py:3-37)."""
import numpy as np


class CompositeOp:
    def __init__(self, *ops_and_starts, shape=None):
        self.ops = [el[0] for el in ops_and_starts]
        self.row_start = [el[1] for el in ops_and_starts]
        self.col_start = [el[2] for el in ops_and_starts]
        n_rows = max([el[1] + el[0].shape[0] for el in ops_and_starts])
        n_cols = max([el[2] + el[0].shape[1] for el in ops_and_starts])
        self.shape = (n_rows, n_cols) if shape is None else shape

    def generic_dot(self, v, dot_name):
        out = np.zeros([self.shape[0]] + list(v.shape[1:]))
        for op, r0, c0 in zip(self.ops, self.row_start, self.col_start):
            out[r0:r0 + op.shape[0]] += getattr(op, dot_name)(v[c0:c0 + op.shape[1]])
        return out

    def nearfield_dot(self, v):
        return self.generic_dot(v, "nearfield_dot")

    def nearfield_no_correction_dot(self, v):
        return self.generic_dot(v, "nearfield_no_correction_dot")

    def dot(self, v):
        return self.generic_dot(v, "dot")

    def farfield_dot(self, v):
        return self.generic_dot(v, "farfield_dot")
