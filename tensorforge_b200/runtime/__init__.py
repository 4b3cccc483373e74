"""Native runtime: nvcc build cache, ctypes launcher binding, device buffers."""
from .build import build_library, BuildError
from .kernel import CompiledKernel, compile_generator, LaunchError
