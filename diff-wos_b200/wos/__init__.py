"""wos -- walk-on-spheres Poisson solver with differential estimators,
B200-native (sm_100a) drop-in for the hot path of diff-wos.

The Python API mirrors the reference package `wos` (scene and solver classes,
solve / walk returning per-point values, gradient solvers); tensors are torch
CUDA tensors and every compute path runs in libwos_b200.so through its C ABI
(include/wos_b200.h).  There is no CPU fallback.
"""
from . import _lib, shapes
from .batch import BatchItem, BatchPlan
from ._lib import (WosError, device_status, get_launch_config, set_launch_config, set_sample_order,
                   set_work_counting, work_counters)
from .scene import BoundarySamplingRecord, ClosestPointRecord, Detector, Intersection, Polyline
from .scene3d import ClosestPointRecord3D, Detector3D, Detector3DY, Scene3D
from .solver import ControlVarianceType, CustomSolver, Sampler, Solver
from .stats import Statistics, merge_solves
from .wos import Baseline, WoS, WoSCUDA
from .wos3d import WoS3D, WoS3DCUDA
from .wos_grad import Ours, OursCUDA
from .wos_grad_3d import Baseline3D, Ours3D
from .baselines import Baseline2, Baseline2CUDA, Baseline23D
from .wos_boundary import WoSBoundary
from .wos_with_source import WoSWithSource, WoSWithSourceCUDA

__all__ = [
    "BoundarySamplingRecord", "ClosestPointRecord", "ClosestPointRecord3D", "ControlVarianceType", "CustomSolver",
    "Detector", "Detector3D", "Detector3DY", "Intersection", "Ours", "Ours3D", "OursCUDA", "Polyline", "Sampler",
    "Scene3D", "Solver", "Statistics", "WoS", "WoS3D", "WoS3DCUDA", "WoSCUDA", "WoSWithSource", "WoSWithSourceCUDA",
    "Baseline", "WosError", "device_status", "get_launch_config", "set_launch_config", "set_sample_order",
    "set_work_counting",
    "work_counters", "merge_solves", "shapes", "BatchItem", "BatchPlan", "WoSBoundary", "Baseline2", "Baseline2CUDA", "Baseline23D", "Baseline3D",
]
