"""The native runtime library (libtfb200_runtime.so): C-ABI entry points built from csrc/."""
import ctypes
import glob
import os

from .build import ARCH_FLAGS, BASE_FLAGS, CSRC, INCLUDE, _run, nvcc

LIB = os.path.join(os.path.dirname(CSRC), 'libtfb200_runtime.so')


def sources():
  return sorted(glob.glob(os.path.join(CSRC, '*.cu')))


def build(force=False):
  srcs = sources()
  newest = max(os.path.getmtime(s) for s in srcs + glob.glob(os.path.join(INCLUDE, '*.h')))
  if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
    return LIB
  tmp = LIB + f'.{os.getpid()}.tmp'
  _run([nvcc()] + ARCH_FLAGS + BASE_FLAGS + [f'-I{INCLUDE}', '-shared'] + srcs + ['-o', tmp, '-lcuda'],
       LIB + '.log')
  os.replace(tmp, LIB)
  return LIB


_lib = None


def load():
  global _lib
  if _lib is None:
    if not os.path.exists(LIB):
      raise RuntimeError(f'native runtime not built: {LIB} (run __graft_entry__.build())')
    _lib = ctypes.CDLL(LIB, mode=ctypes.RTLD_LOCAL)
  return _lib
