"""Elastic Green's-function catalogue: names and attributes as in the
reference's tectosaur/kernels/__init__.py:3-258 (the formulas themselves live
in the CUDA sources, csrc/pair_math.cuh and csrc/farfield.cu).

scale_type is the power of length the kernel scales with (used to undo a
mesh rescaling, ops/sparse_farfield_op.py:89-94); multipole_dim is the number
of multipole moments the treecode keeps per order.
"""
import collections

Kernel = collections.namedtuple(
    "Kernel",
    ["name", "spatial_dim", "tensor_dim", "needs_obsn", "needs_srcn", "scale_type",
     "sm_power", "flip_negate", "surf_curl_obs", "surf_curl_src", "multipole_dim", "id"])

elastic_kernels = {
    "elasticU3": Kernel("elasticU3", 3, 3, False, False, -3, 1, False, False, False, 7, 0),
    "elasticT3": Kernel("elasticT3", 3, 3, False, True, -2, 0, True, False, False, 0, 1),
    "elasticA3": Kernel("elasticA3", 3, 3, True, False, -2, 0, True, False, False, 0, 2),
    "elasticH3": Kernel("elasticH3", 3, 3, True, True, -1, -1, False, False, False, 0, 3),
}
regularized_elastic_kernels = {
    "elasticRT3": Kernel("elasticRT3", 3, 3, False, True, -2, 0, True, False, True, 10, 4),
    "elasticRA3": Kernel("elasticRA3", 3, 3, True, False, -2, 0, True, True, False, 7, 5),
    "elasticRH3": Kernel("elasticRH3", 3, 3, True, True, -1, 1, False, True, True, 22, 6),
}
kernels = dict(elastic_kernels)
kernels.update(regularized_elastic_kernels)
