"""motionest: B200-native SAMER/DISORDER joint motion-corrected reconstruction.

Drop-in for the reference's hot-path API (chiew-group/motion-estimation):
RigidTransformCudaOptimzied, RigidTransformDerivativeCuda, estimate_image_cg,
estimate_transform, JointRecon, pyramid_reconstruction, compute_transform_grids_voxel.
All compute runs in libmotionest.so (hand-written sm_100a CUDA); there is no CPU fallback.
"""
from .transform import RigidTransformCudaOptimzied, RigidTransformDerivativeCuda  # noqa: F401
from .utils import compute_transform_grids_voxel  # noqa: F401

__all__ = ["RigidTransformCudaOptimzied", "RigidTransformDerivativeCuda",
           "compute_transform_grids_voxel"]
