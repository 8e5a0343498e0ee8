"""B200-native explicit meshfree step (MEGA / XieZhengTing/Taylor hot path).

The compute path is libmega_gpu.so (hand-written sm_100a CUDA); this package
holds its ctypes binding, a host-side mirror of the reference's subroutine
interface, the synthetic case generators and the build recipe.
"""
from . import _lib, cases  # noqa: F401
from .mega import (Mega, bin_search, constitution, construct_fint, hughes_winget,  # noqa: F401
                   rk_shapes, rotate_tensor)
