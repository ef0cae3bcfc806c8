"""B200-native SPH cutting step (iwf_mfree_gpu_3d's leap_frog::step) behind a C ABI.

``libmfree.so`` (built from ``csrc/`` by ``build.py``) holds the CUDA kernels for
sm_100a and the C++ host code; ``api.Simulation`` binds it; ``scenes`` builds
the cutting scenes.
"""
from . import scenes  # noqa: F401

__all__ = ["scenes", "api", "build"]
