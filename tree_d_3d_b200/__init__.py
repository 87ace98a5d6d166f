"""B200-native field evaluation of charges in a plane (tree-d-3d's FlatQuadtree).

``FlatQuadtree`` (build, Barnes-Hut ``evaluate``, FMM ``fmm``/``fmm_at``) and
``direct_field`` for the ``"coulomb"`` and ``"log"`` kernels, with the reference's
Python API on PyTorch CUDA tensors; every numeric step runs in hand-written sm_100a
kernels of libtreed3d.so through the C ABI of include/treed3d.h.
"""

from tree_d_3d_b200.constants import K_E
from tree_d_3d_b200.flat_tree import (
    COULOMB_ORDER,
    LOG_ORDER,
    MAX_ORDER,
    FlatNode,
    FlatQuadtree,
    direct_field,
)
from tree_d_3d_b200.quad import Quad
from tree_d_3d_b200.strip import GroundedStripField

__version__ = "0.1.0"

__all__ = [
    "K_E",
    "COULOMB_ORDER",
    "LOG_ORDER",
    "MAX_ORDER",
    "FlatNode",
    "FlatQuadtree",
    "GroundedStripField",
    "Quad",
    "direct_field",
]
