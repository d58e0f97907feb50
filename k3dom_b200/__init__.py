"""k3dom_b200: B200-native K3DOM / DS-PHD/MIB map-and-track update behind a C ABI.

The compute path is libk3dom_b200.so (hand-written sm_100a CUDA, built with
`python -m k3dom_b200.build`); this package holds the Python mirror of the reference's
update API (dom.py), the ctypes binding (_native.py) and the synthetic scene generator
(scene.py).
"""
from .dom import (DOM, GRIDCELL_DTYPE, BatchDOM, MAPPOINT_DTYPE, debug_draws, make_params, node_config_from_yaml,  # noqa: F401
                  params_default, params_from_yaml, rotation_from_quaternion)

__all__ = ["BatchDOM", "DOM", "GRIDCELL_DTYPE", "MAPPOINT_DTYPE", "debug_draws", "make_params", "node_config_from_yaml",
           "params_default", "params_from_yaml", "rotation_from_quaternion"]
