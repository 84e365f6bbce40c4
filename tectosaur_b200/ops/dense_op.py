"""Dense operator wrapper (reference: tectosaur/ops/dense_op.py:1-18)."""
import numpy as np


class DenseOp:
    def __init__(self, mat):
        self.mat = mat
        self.shape = mat.shape

    def dot(self, v):
        return self.mat.dot(v)

    def nearfield_dot(self, v):
        return self.dot(v)

    def nearfield_no_correction_dot(self, v):
        return self.dot(v)

    def farfield_dot(self, v):
        return np.zeros(self.shape[0])
