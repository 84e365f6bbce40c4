"""Sum of operators (reference: tectosaur/ops/sum_op.py:1-16).

When every term has a device apply (the integral operators, MassOp, MultOp
of those), ``dot`` of a host array copies it to the device once, applies the
terms into one output buffer (the first writes, the rest accumulate) and
copies the sum back once; otherwise each term's ``dot`` runs as in the
reference.
"""
import numpy as np

from ..util import device


def fixed_float_type(ops):
    """The widest float_type among ops that fix one, or None when none does
    (MassOp applies in the precision of its input)."""
    fts = [np.dtype(op.float_type) for op in ops if getattr(op, "float_type", None) is not None]
    return max(fts, key=lambda f: f.itemsize) if fts else None


class SumOp:
    def __init__(self, ops):
        self.ops = ops
        self.shape = ops[0].shape

    def on_device(self):
        return all(hasattr(op, "dot_device") for op in self.ops)

    @property
    def float_type(self):
        return fixed_float_type(self.ops)

    def dot_device(self, x, y, stream=None, accumulate=False):
        """y (+)= sum_k op_k x on device tensors."""
        for k, op in enumerate(self.ops):
            op.dot_device(x, y, stream=stream, accumulate=bool(accumulate) or k > 0)
        return y

    def dot_panel_device(self, X, Y, stream=None, accumulate=False):
        for k, op in enumerate(self.ops):
            op.dot_panel_device(X, Y, stream=stream, accumulate=bool(accumulate) or k > 0)
        return Y

    def nearfield_dot(self, v):
        return sum([op.nearfield_dot(v) for op in self.ops])

    def nearfield_no_correction_dot(self, v):
        return sum([op.nearfield_no_correction_dot(v) for op in self.ops])

    def dot(self, v):
        if self.on_device() and (device.is_device_tensor(v) or device.cuda_available()):
            return device.host_or_device_apply(self, v, self.float_type or np.float64)
        return sum([op.dot(v) for op in self.ops])

    def farfield_dot(self, v):
        return sum([op.farfield_dot(v) for op in self.ops])
