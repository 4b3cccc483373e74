"""Build and run the reference's own generated kernels on the host (OpenMP backend).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Recipe: import the reference generator from the read-only source tree, generate a
chain with `Context(arch='sm_100', backend='omptarget', fp_type=...)`, wrap the emitted
kernel + launcher with a small C entry point and compile it together with the
reference's `tensorforge/include/tensorforge_aux_target.cpp` using
`g++ -O3 -march=native -fopenmp`. All generated sources and binaries go to oracle/_ref/.
The compiled libraries are then loaded with ctypes (this part needs no source tree, so
it also runs on a machine that only received the built files).

Caveats from the reference: the emitted region is `nowait`,
so the entry point ends with `#pragma omp taskwait`; element counts must be a multiple
of the kernel's elements-per-block, because the emitted barrier sits inside the
element guard (target_lexic.py:147-168, generator.py:145-146) - callers pad N and mask
the padding with flags; the launcher rejects a null stream (target_lexic.py:182-187).
"""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, '_ref')
# The read-only reference checkout this recipe reads (generator sources and
# tensorforge/include). Set TFB_REFERENCE_ROOT to use another checkout; every other
# script that needs the reference tree takes the path from here.
DEFAULT_REFERENCE_ROOT = '/root/reference'
REFERENCE_ROOT = os.environ.get('TFB_REFERENCE_ROOT', DEFAULT_REFERENCE_ROOT)


def reference_present():
  """True when the reference generator sources are readable at REFERENCE_ROOT."""
  return os.path.isdir(os.path.join(REFERENCE_ROOT, 'tensorforge'))


def _reference_ns():
  if REFERENCE_ROOT not in sys.path:
    sys.path.insert(0, REFERENCE_ROOT)
  from oracle.cases import ns_from_module
  return ns_from_module('tensorforge')


def generate(descr_builder, fp='float', backend='omptarget'):
  """Run the reference generator; returns (kernel, launcher, header, base_name, mults_per_block)."""
  ns = _reference_ns()
  from tensorforge.common.context import Context
  from tensorforge.generators.generator import Generator
  descrs = descr_builder(ns)
  ftype = ns.FloatingPointType.FLOAT if fp == 'float' else ns.FloatingPointType.DOUBLE
  g = Generator(descrs, Context(arch='sm_100', backend=backend, fp_type=ftype))
  g.generate()
  mults = g._shr_mem_obj.get_mults_per_block()
  return g.get_kernel(), g.get_launcher(), g.get_header(), g.get_base_name(), mults


def parse_params(header):
  """Parameter list of an emitted launcher prototype: [(type, name)]."""
  inner = header[header.index('(') + 1: header.rindex(')')]
  out = []
  for p in inner.split(','):
    p = p.split('=')[0].strip()
    m = re.match(r'^(.*?)([A-Za-z_][A-Za-z0-9_]*)$', p)
    out.append((m.group(1).strip(), m.group(2)))
  return out


def _wrapper(header, base, fp):
  """C entry point `tfref_run(void** ptrs, const unsigned* offs, const double* scalars,
  size_t n, unsigned* flags)` that calls the launcher with symbols in ABI order."""
  params = parse_params(header)
  args = []
  i_ptr = i_off = i_sc = 0
  for typ, name in params:
    if name in ('numElements',):
      args.append('n')
    elif name == 'flags':
      args.append('flags')
    elif name == 'streamPtr':
      args.append('&stream')
    elif name.endswith('_extraOffset'):
      args.append(f'offs[{i_off}]')
      i_off += 1
    elif '*' in typ:
      args.append(f'({typ})ptrs[{i_ptr}]')
      i_ptr += 1
    else:
      args.append(f'({typ})scalars[{i_sc}]')
      i_sc += 1
  return (
    'extern "C" int tfref_run(void** ptrs, const unsigned* offs, const double* scalars, '
    'size_t n, unsigned* flags) {\n'
    '  int stream = 0;\n'
    f'  launcher_{base}({", ".join(args)});\n'
    '  #pragma omp taskwait\n'
    '  return 0;\n'
    '}\n')


def generate_source(tag, descr_builder, fp='float'):
  """Run the reference generator for one case and write oracle/_ref/<tag>.cpp and .meta
  (the metadata file is written only once the library is built)."""
  os.makedirs(REF_OUT, exist_ok=True)
  kernel, launcher, header, base, mults = generate(descr_builder, fp)
  src = os.path.join(REF_OUT, f'{tag}.cpp')
  with open(src, 'w') as f:
    f.write('#include <omp.h>\n#include <cstddef>\n#include <stdexcept>\n#include <cmath>\n')
    f.write('#include "tensorforge_aux.h"\n\n')
    f.write(kernel + '\n' + launcher + '\n' + _wrapper(header, base, fp))
  with open(os.path.join(REF_OUT, f'{tag}.pending'), 'w') as f:
    f.write(f'{base}\n{mults}\n{header}')
  return src


def compile_source(tag, opt='-O3'):
  """Compile oracle/_ref/<tag>.cpp with the reference's host runtime into <tag>.so."""
  src = os.path.join(REF_OUT, f'{tag}.cpp')
  so = os.path.join(REF_OUT, f'{tag}.so')
  inc = os.path.join(REFERENCE_ROOT, 'tensorforge', 'include')
  aux = os.path.join(inc, 'tensorforge_aux_target.cpp')
  tmp = so + f'.{os.getpid()}.tmp'
  cmd = ['g++', opt, '-march=native', '-fopenmp', '-fPIC', '-shared', f'-I{inc}', src, aux, '-o', tmp]
  subprocess.run(cmd, check=True)
  os.replace(tmp, so)
  os.replace(os.path.join(REF_OUT, f'{tag}.pending'), os.path.join(REF_OUT, f'{tag}.meta'))
  return so


def build(tag, descr_builder, fp='float', opt='-O3', force=False):
  """Generate + compile one reference OpenMP kernel into oracle/_ref/<tag>.so."""
  so = os.path.join(REF_OUT, f'{tag}.so')
  meta = os.path.join(REF_OUT, f'{tag}.meta')
  if os.path.exists(so) and os.path.exists(meta) and not force:
    return so
  generate_source(tag, descr_builder, fp)
  return compile_source(tag, opt)


class RefKernel:
  """ctypes handle on one built reference kernel."""

  def __init__(self, tag):
    so = os.path.join(REF_OUT, f'{tag}.so')
    with open(os.path.join(REF_OUT, f'{tag}.meta')) as f:
      lines = f.read().split('\n', 2)
    self.base_name = lines[0]
    self.mults_per_block = int(lines[1])
    self.header = lines[2]
    self.lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    self.fn = self.lib.tfref_run
    self.fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    self.fn.restype = ctypes.c_int

  def run(self, layouts, host_buffers, n, scalars=None):
    """host_buffers: {name: np.ndarray (float32/64, modified in place)}.

    The element count is padded to a multiple of the kernel's elements per block with
    dummy elements that compute on scratch copies (flags cannot mask them: the emitted
    barrier sits inside the flags guard as well, so masked threads would never reach it).
    """
    mult = self.mults_per_block
    n_pad = ((n + mult - 1) // mult) * mult
    extra = n_pad - n
    ptrs, offs, scs = [], [], []
    keep, copy_back = [], []
    for lay in layouts:
      if lay.kind == 'scalar':
        scs.append(float(scalars[lay.name]))
        continue
      buf = host_buffers[lay.name]
      if lay.kind == 'ptr':
        scratch = np.zeros(max(1, extra) * lay.slot, dtype=buf.dtype)
        keep.append(scratch)
        arr = np.zeros(n_pad, dtype=np.uint64)
        arr[:n] = buf.ctypes.data + (lay.starts - lay.extra_offset) * buf.itemsize
        arr[n:] = scratch.ctypes.data + np.arange(extra, dtype=np.uint64) * lay.slot * buf.itemsize
        keep.append(arr)
        ptrs.append(arr.ctypes.data)
        offs.append(lay.extra_offset)
      elif lay.kind == 'strided':
        need = n_pad * lay.slot + lay.extra_offset + 4
        if extra > 0 and need > buf.size:
          big = np.zeros(need, dtype=buf.dtype)
          big[:buf.size] = buf
          keep.append(big)
          copy_back.append((buf, big, n * lay.slot + lay.extra_offset))
          ptrs.append(big.ctypes.data)
        else:
          ptrs.append(buf.ctypes.data)
        offs.append(lay.extra_offset)
      else:
        ptrs.append(buf.ctypes.data)
    p_arr = (ctypes.c_void_p * max(1, len(ptrs)))(*ptrs)
    o_arr = (ctypes.c_uint * max(1, len(offs)))(*offs)
    s_arr = (ctypes.c_double * max(1, len(scs)))(*scs)
    self.fn(p_arr, o_arr, s_arr, n_pad, None)
    for buf, big, span in copy_back:
      buf[:span] = big[:span]
    return host_buffers
