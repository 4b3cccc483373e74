"""Load a generated launcher and call it through its C ABI (ctypes), with torch buffers.

The call goes to `tfb_launch_<kernel name>(...)`, the `extern "C"` twin that every
generated library exports beside the reference-named C++ launcher
`launcher_<kernel name>(...)`: the same parameter list, with the launch's CUDA status
as the return value (ctypes cannot bind a C++-mangled name). Pointer arguments
accept torch tensors (their `data_ptr()`), raw integer addresses or None; pointer
arrays for PTR_BASED operands are device tensors of int64 addresses; `streamPtr`
accepts a torch.cuda.Stream, a raw cudaStream_t or None (the current torch stream).
"""
import ctypes
import os

from .build import build_library

_CTYPES = {
  'float': ctypes.c_float, 'double': ctypes.c_double, 'unsigned': ctypes.c_uint,
  'size_t': ctypes.c_size_t, 'int': ctypes.c_int,
}


class LaunchError(RuntimeError):
  pass


def _ctype(c_type):
  if '*' in c_type:
    return ctypes.c_void_p
  base = c_type.replace('const ', '').strip()
  return _CTYPES[base]


def _ptr(x):
  if x is None:
    return None
  if isinstance(x, int):
    return x
  if hasattr(x, 'data_ptr'):
    return int(x.data_ptr())
  raise TypeError(f'cannot pass {type(x).__name__} as a pointer')


def require_cuda():
  import torch
  if not torch.cuda.is_available():
    raise LaunchError('no CUDA device: generated kernels run on the GPU only (no CPU fallback)')


class CompiledKernel:
  """A built generator output bound to its launcher symbol."""

  def __init__(self, generator, so_path=None):
    self.generator = generator
    self.name = generator.get_base_name()
    self.params = generator.abi_params()
    self.so_path = so_path or build_library(generator.get_source())
    self._lib = None

  def _load(self):
    if self._lib is None:
      if not os.path.exists(self.so_path):
        raise LaunchError(f'kernel library missing: {self.so_path}')
      self._lib = ctypes.CDLL(self.so_path, mode=ctypes.RTLD_LOCAL)
      fn = getattr(self._lib, f'tfb_launch_{self.name}')
      fn.argtypes = [_ctype(t) for t, _ in self.params]
      fn.restype = ctypes.c_int
      self._fn = fn
    return self._fn

  def address(self):
    """Address of the status-returning entry point (for C callers that receive a function
    pointer)."""
    self._load()
    return ctypes.cast(self._fn, ctypes.c_void_p).value

  def __call__(self, *args, **kwargs):
    """Call with arguments in ABI order (positional) or by parameter name.

    `numElements` is required; `flags` and `streamPtr` default to nullptr / the
    current torch stream. Extra offsets default to 0.
    """
    import torch
    require_cuda()
    fn = self._load()
    names = [n for _, n in self.params]
    values = dict(zip(names, args))
    values.update(kwargs)
    if 'numElements' not in values:
      raise TypeError('numElements is required')
    values.setdefault('flags', None)
    if values.get('streamPtr') is None:
      values['streamPtr'] = torch.cuda.current_stream().cuda_stream
    out = []
    for (c_type, name) in self.params:
      v = values.get(name)
      if name.endswith('_extraOffset') and v is None:
        v = 0
      if '*' in c_type:
        if name == 'streamPtr' and hasattr(v, 'cuda_stream'):
          v = v.cuda_stream
        out.append(_ptr(v))
      else:
        if v is None:
          raise TypeError(f'missing argument {name}')
        out.append(v)
    status = fn(*out)
    if status != 0:
      raise LaunchError(f'launcher_{self.name} failed with CUDA error {status}')


def compile_generator(generator):
  """Build (or fetch from the cache) and bind a generated kernel."""
  return CompiledKernel(generator)
