"""kinectfusion_b200: KinectFusion's per-frame pipeline on NVIDIA B200 (sm_100a).

The compute lives in libkf_b200.so (hand-written CUDA behind the C ABI of
include/kf_b200.h); this package is the Python host mirror of the reference's
Pipeline / PyramidSource / ProjectiveIcpTracker interfaces over that ABI.
"""

from . import abi, learned, pipeline_set, synthetic, tum  # noqa: F401
from .pipeline import (ICP_ITERATIONS, Batch, Pipeline, PipelinedReconstruction, ProjectiveIcpTracker,  # noqa: F401
                       PyramidSource, Reconstruction, SurfaceMaps, default_depth_options, default_icp_options,
                       device_available, pipeline_config)

from .pipeline_set import AblationStats, PipelineComparison, PipelineSet, SetReconstruction  # noqa: F401

__all__ = ["abi", "learned", "pipeline_set", "synthetic", "tum", "Batch", "PipelineSet", "SetReconstruction",
           "PipelineComparison", "AblationStats", "Pipeline", "PyramidSource", "ProjectiveIcpTracker", "Reconstruction", "PipelinedReconstruction",
           "SurfaceMaps", "pipeline_config", "default_depth_options", "default_icp_options",
           "device_available", "ICP_ITERATIONS"]
