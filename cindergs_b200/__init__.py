"""cindergs_b200: the CinderGS four-stage Gaussian-splat pipeline (tet cage
deformation, EWA projection with inverse-ray SH, tile binning and sort, tile
compositing) as hand-written sm_100a CUDA behind a C ABI (include/cgs.h).

The Python modules are the host side of that ABI: scene and cage set-up and a
mirror of the reference crate's GpuPipelineState API. All per-frame compute
runs in ``_lib/libcindergs.so``; there is no CPU fallback.
"""
from .camera import CameraUniforms, CompositorUniforms, look_at_lh, orbit_camera
from .cage import Cage, CageScene, CageSpringSimulator, TetMesh, UNBOUND
from .pipeline import (GpuPipelineState, GpuStageTimings, exclusive_scan_u32,
                       radix_sort_u32_pairs, radix_sort_u64_pairs, scene_fingerprint)
from .mvc import PolyCageMesh
from . import ply
from .scene import GaussianSceneSoa, QuantizedGaussianSceneSoa, fibonacci_cluster, random_scene

__all__ = [
    "CameraUniforms", "CompositorUniforms", "look_at_lh", "orbit_camera", "Cage", "CageScene",
    "CageSpringSimulator", "TetMesh", "UNBOUND", "GpuPipelineState", "GpuStageTimings",
    "exclusive_scan_u32", "radix_sort_u32_pairs", "radix_sort_u64_pairs", "scene_fingerprint",
    "GaussianSceneSoa", "QuantizedGaussianSceneSoa", "fibonacci_cluster", "random_scene", "PolyCageMesh", "ply",
]
