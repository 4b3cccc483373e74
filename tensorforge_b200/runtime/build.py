"""Compile generated sources for sm_100a into shared libraries, cached in-tree.

Every library is built with `nvcc -gencode arch=compute_100a,code=sm_100a` and linked
with the runtime helpers (csrc/tensorforge_aux.cu). Libraries are keyed by a hash of
the source text and the compiler flags and stored under `tensorforge_b200/_kcache/`
(override with TFB_KCACHE), so a build done on a machine without a GPU is reused
unchanged by the machine that runs it.
"""
import hashlib
import os
import shutil
import subprocess
import threading

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO = os.path.dirname(PKG)
INCLUDE = os.path.join(REPO, 'include')
CSRC = os.path.join(PKG, 'csrc')
CACHE = os.environ.get('TFB_KCACHE', os.path.join(PKG, '_kcache'))

ARCH_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a']
BASE_FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr']

_lock = threading.Lock()


class BuildError(RuntimeError):
  pass


def nvcc():
  path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
  if not os.path.exists(path):
    raise BuildError('nvcc not found: the CUDA toolkit is required to build generated kernels')
  return path


def _run(cmd, log):
  proc = subprocess.run(cmd, capture_output=True, text=True)
  with open(log, 'w') as f:
    f.write(' '.join(cmd) + '\n' + proc.stdout + proc.stderr)
  if proc.returncode != 0:
    raise BuildError(f'nvcc failed ({proc.returncode}); see {log}\n{proc.stderr[-4000:]}')
  return proc


def aux_object():
  """The runtime helper object, built once per cache directory."""
  os.makedirs(CACHE, exist_ok=True)
  src = os.path.join(CSRC, 'tensorforge_aux.cu')
  with open(src, 'rb') as f:
    h = hashlib.sha1(f.read() + ' '.join(ARCH_FLAGS + BASE_FLAGS).encode()).hexdigest()[:16]
  obj = os.path.join(CACHE, f'tensorforge_aux_{h}.o')
  if not os.path.exists(obj):
    tmp = obj + f'.{os.getpid()}.tmp.o'
    _run([nvcc()] + ARCH_FLAGS + BASE_FLAGS + [f'-I{INCLUDE}', '-c', src, '-o', tmp], obj + '.log')
    os.replace(tmp, obj)
  return obj


# extra flag token (never passed to nvcc): build without -lineinfo, for libraries that are
# timed but never profiled (the autotuner's variant libraries are 2.5x smaller without it)
NO_LINEINFO = '--tfb-no-lineinfo'


def _nvcc_flags(extra_flags):
  base = [f for f in BASE_FLAGS if not (f == '-lineinfo' and NO_LINEINFO in extra_flags)]
  return base + [f for f in extra_flags if f != NO_LINEINFO]


def source_key(source, extra_flags=()):
  return hashlib.sha1((source + '\0' + ' '.join(ARCH_FLAGS + BASE_FLAGS + list(extra_flags))).encode()).hexdigest()[:20]


def library_path(source, extra_flags=()):
  return os.path.join(CACHE, f'tfb_{source_key(source, extra_flags)}.so')


def build_library(source, extra_flags=(), verbose_ptxas=False):
  """Compile `source` (a complete .cu translation unit) and return the .so path."""
  so = library_path(source, extra_flags)
  if os.path.exists(so):
    return so
  with _lock:  # the shared helper object is built once; libraries build concurrently
    os.makedirs(CACHE, exist_ok=True)
    aux = aux_object()
  # per-process, per-thread temporaries + atomic rename: concurrent builders of the same
  # source (threads or processes) each produce a complete file and the last rename wins
  tag = f'{os.getpid()}.{threading.get_ident()}'
  cu = so[:-3] + f'.{tag}.cu'
  with open(cu, 'w') as f:
    f.write(source)
  flags = _nvcc_flags(extra_flags) + (['-Xptxas', '-v'] if verbose_ptxas else [])
  tmp = so + f'.{tag}.tmp.so'
  try:
    _run([nvcc()] + ARCH_FLAGS + flags + [f'-I{INCLUDE}', '-shared', cu, aux, '-o', tmp, '-lcuda'],
         so[:-3] + '.log')
    os.replace(tmp, so)
    os.replace(cu, so[:-3] + '.cu')
  finally:
    for path in (cu, tmp):
      if os.path.exists(path):
        os.remove(path)
  return so


def is_cached(source, extra_flags=()):
  return os.path.exists(library_path(source, extra_flags))
