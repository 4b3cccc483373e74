"""tensorforge_b200: a B200-native (sm_100a) generator of batched small-tensor contraction kernels.

Drop-in for TensorForge's Python frontend and its CUDA backend's launcher ABI.
"""
from .interop import *  # noqa: F401,F403
