"""Scaled operator (reference: tectosaur/ops/neg_op.py:1-21).

With a device apply underneath, ``dot_device`` scales on the device: the
wrapped operator writes into y (or a scratch buffer when accumulating) and
one elementwise pass applies the factor.
"""
import numpy as np

from ..util import device


class MultOp:
    def __init__(self, op, factor):
        self.op = op
        self.shape = op.shape
        self.factor = factor

    def on_device(self):
        return hasattr(self.op, "dot_device")

    @property
    def float_type(self):
        from .sum_op import fixed_float_type
        return fixed_float_type([self.op])

    def _scaled(self, apply, y, stream, accumulate):
        t = device.torch()
        ctx = t.cuda.stream(stream) if stream is not None else t.cuda.stream(
            t.cuda.current_stream())
        if not accumulate:
            apply(y)
            with ctx:
                y.mul_(self.factor)
            return y
        tmp = t.empty_like(y)
        apply(tmp)
        with ctx:
            y.add_(tmp, alpha=self.factor)
        return y

    def dot_device(self, x, y, stream=None, accumulate=False):
        """y (+)= factor * op x on device tensors."""
        return self._scaled(lambda out: self.op.dot_device(x, out, stream=stream), y, stream,
                            accumulate)

    def dot_panel_device(self, X, Y, stream=None, accumulate=False):
        return self._scaled(lambda out: self.op.dot_panel_device(X, out, stream=stream), Y,
                            stream, accumulate)

    def nearfield_dot(self, v):
        return self.factor * self.op.nearfield_dot(v)

    def nearfield_no_correction_dot(self, v):
        return self.factor * self.op.nearfield_no_correction_dot(v)

    def dot(self, v):
        if self.on_device() and (device.is_device_tensor(v) or device.cuda_available()):
            return device.host_or_device_apply(self, v, self.float_type or np.float64)
        return self.factor * self.op.dot(v)

    def farfield_dot(self, v):
        return self.factor * self.op.farfield_dot(v)


def NegOp(op):
    return MultOp(op, -1)
