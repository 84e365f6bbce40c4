"""tectosaur_b200: the elastic-BEM operator apply of tectosaur, B200-native.

Drop-in for the reference's ``tectosaur.ops`` API: the same operator classes,
constructor signatures and ``dot`` / ``nearfield_dot`` / ``farfield_dot``
methods, computed by hand-written sm_100a CUDA kernels in libtct_b200.so
(C ABI: include/tct_b200.h).
"""
from .mesh.mesh_gen import make_rect
from .ops.mass_op import MassOp
from .ops.sum_op import SumOp
from .ops.neg_op import NegOp, MultOp
from .ops.composite_op import CompositeOp
from .ops.dense_op import DenseOp
from .ops.sparse_integral_op import RegularizedSparseIntegralOp
from .ops.sparse_farfield_op import TriToTriDirectFarfieldOp
from .ops.dense_integral_op import RegularizedDenseIntegralOp, farfield_tris
from .farfield import farfield_pts_direct
from .interior import InteriorOp
from .kernels import kernels

__all__ = [
    "make_rect", "MassOp", "SumOp", "NegOp", "MultOp", "CompositeOp", "DenseOp",
    "RegularizedSparseIntegralOp", "TriToTriDirectFarfieldOp", "RegularizedDenseIntegralOp",
    "farfield_tris", "farfield_pts_direct", "InteriorOp", "kernels",
]
