"""lightpropagation_b200 -- B200-native MCML photon transport through triangle meshes.

Drop-in for the hot path of LightPropagation (the MCLightPropagation OpenCL kernel
and its CalculatePropagation launcher).  The compute path is liblpcuda.so
(hand-written CUDA for sm_100a) behind the C ABI in include/lpcuda.h.
"""
from .propagation import CalculatePropagation, ImageData, Simulation, philox_blocks  # noqa: F401
from .batch import Batch, Instance  # noqa: F401
from . import meshes, workloads  # noqa: F401

__all__ = ["CalculatePropagation", "ImageData", "Simulation", "Batch", "Instance", "philox_blocks", "meshes",
           "workloads"]
