"""Exhaustive autotuning: every variant of a chain is generated, built and timed on the GPU.

All variants of one chain go into one translation unit (one nvcc invocation); each variant
keeps the chain's launcher ABI under its own kernel name (`<md5 name>_v<i>`). Requested
variants that the planner realises identically (a constant-memory A that falls back to
shared memory, a column program that does not fit and falls back to the generic plan) are
kept once. `build_chain` is pure host work and returns a picklable `ChainBuild`, so a
process pool can compile while the GPU process measures. Timings are cached per (GPU
name and driver, variant space, chain signature) as JSON, so interrupted tuning runs resume
where they stopped.
"""
import hashlib
import json
import os
from dataclasses import dataclass
from typing import List, Tuple

from ..common.basic_types import FloatingPointType
from ..common.context import Context, Options
from ..generators.generator import Generator
from ..codegen import PRELUDE
from ..runtime.build import build_library
from .chains import build_descriptors, ChainSpec
from .variants import variant_space, effective_variant, features


def _ns():
  from types import SimpleNamespace
  from ..common.matrix.tensor import Tensor, SubTensor
  from ..common.matrix.spp import ListSPP
  from ..common.basic_types import Addressing
  from ..generators.descriptions import MultilinearDescr
  from ..common.aux import generate_tmp_tensor
  return SimpleNamespace(Tensor=Tensor, SubTensor=SubTensor, ListSPP=ListSPP, Addressing=Addressing,
                         MultilinearDescr=MultilinearDescr, generate_tmp_tensor=generate_tmp_tensor)


def make_generator(spec, variant=None, name=None, fp=FloatingPointType.FLOAT):
  g = Generator(build_descriptors(spec, _ns()), Context('sm_100a', 'cuda', fp, Options(variant=variant)))
  if name is not None:
    g.register()
    g.set_kernel_name(name)
  g.generate()
  return g


@dataclass
class ChainBuild:
  """Everything the measuring process needs about one chain's variant library."""
  spec: ChainSpec
  so_path: str
  params: list                  # launcher ABI [(c type, name)], shared by all variants
  buffers: List[Tuple[str, int]]  # (ABI name, values to allocate) per tensor argument
  dest: str                     # ABI name of the output tensor
  names: List[str]              # launcher kernel name per variant
  variants: List[dict]          # realised variant per entry of `names`
  feats: List[list]             # cost-model features per variant
  default: int                  # index of the variant the planner picks on its own


def variant_library(spec):
  """(source, [(realised variant, generator)], default index) for every distinct variant."""
  base = make_generator(spec)
  default_key = base.get_plan().key()
  seen = {}
  gens = []
  parts = [PRELUDE]
  for v in variant_space(base.get_chain()):
    probe = make_generator(spec, v)
    key = probe.get_plan().key()
    if key in seen:
      continue
    seen[key] = len(gens)
    g = make_generator(spec, v, f'{base.get_base_name()}_v{len(gens)}')
    gens.append((effective_variant(g.get_plan()), g))
    parts.append(g._emitted.extra_prelude + g.get_kernel() + '\n' + g.get_launcher() + '\n')
  if default_key not in seen:
    g = make_generator(spec, None, f'{base.get_base_name()}_v{len(gens)}')
    seen[default_key] = len(gens)
    gens.append((effective_variant(g.get_plan()), g))
    parts.append(g._emitted.extra_prelude + g.get_kernel() + '\n' + g.get_launcher() + '\n')
  return ''.join(parts), gens, seen[default_key]


def buffer_sizes(generator, batch):
  """[(ABI name, values)] per tensor argument and the name of the written one."""
  out, dest = [], None
  for t, _ in generator.abi_symbols():
    size = t.spp.count_nz() if t.addressing.name == 'NONE' else batch * t.get_real_volume()
    out.append((t.name, max(1, int(size))))
    if t.direction.name != 'SOURCE':
      dest = t.name
  return out, dest


def build_chain(spec, extra_flags=(), compile=True):
  """Generate and compile all variants of `spec` (host only; safe in a worker process).

  With compile=False only the record is made (so_path None): for chains whose timings are
  already cached.
  """
  src, gens, default = variant_library(spec)
  so = build_library(src, extra_flags) if compile else None
  g0 = gens[0][1]
  return ChainBuild(spec, so, g0.abi_params(), *buffer_sizes(g0, spec.batch),
                    [g.get_base_name() for _, g in gens], [v for v, _ in gens],
                    [features(gens[0][1].get_chain(), v, spec.batch) for v, g in gens], default)


class _Abi:
  """Just enough of a generator for CompiledKernel to bind a launcher by name."""

  def __init__(self, name, params):
    self._name, self._params = name, params

  def get_base_name(self):
    return self._name

  def abi_params(self):
    return self._params

  def get_source(self):
    raise RuntimeError('prebuilt tuning library')


def gpu_signature():
  """'<device name>_drv<driver version>': tuning results are only valid for both."""
  import torch
  try:
    import pynvml
    pynvml.nvmlInit()
    drv = pynvml.nvmlSystemGetDriverVersion()
    drv = drv.decode() if isinstance(drv, bytes) else drv
  except Exception:  # NVML missing: key on the device name alone
    drv = 'unknown'
  return f'{torch.cuda.get_device_name()}_drv{drv}'.replace(' ', '_')


def is_cached(cache, spec, gpu):
  return os.path.exists(_cache_path(cache, spec, gpu))


def _cache_path(cache, spec, gpu):
  from .variants import space_signature
  h = hashlib.sha1(spec.key().encode()).hexdigest()[:16]
  return os.path.join(cache, gpu, f'space_{space_signature()}', f'{h}.json')


def measure_chain(cb: ChainBuild, cache=None, reps=3, warmup=1, check_tol=1e-3, slow_ms=100.0):
  """Time every variant of a built chain on the current GPU.

  Each variant is launched `warmup` times, then timed `reps` times with CUDA events on
  the current stream (minimum kept). Every variant's output is compared with the
  planner default's output (max-norm relative difference); a variant above `check_tol`
  is recorded with `ok: false` and never counted as a candidate, and so is a variant
  whose launch the device rejects. Returns a list of {'variant', 'ms', 'ok', 'err'} in
  variant order.
  """
  import torch
  from ..runtime.kernel import CompiledKernel, LaunchError
  path = _cache_path(cache, cb.spec, gpu_signature()) if cache else None
  if path and os.path.exists(path):
    with open(path) as f:
      return json.load(f)['results']
  gen = torch.Generator(device='cuda')
  gen.manual_seed(cb.spec.seed)
  bufs = {n: torch.rand(size, device='cuda', generator=gen) * 2 - 1 for n, size in cb.buffers}
  out_name = cb.dest
  stream = torch.cuda.current_stream()
  kernels = [CompiledKernel(_Abi(n, cb.params), cb.so_path) for n in cb.names]

  def run(k):
    k(numElements=cb.spec.batch, **bufs)

  run(kernels[cb.default])
  ref = bufs[out_name].clone()
  scale = float(ref.abs().max()) or 1.0
  def timed(k):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    run(k)
    e.record(stream)
    e.synchronize()
    return s.elapsed_time(e)

  results = []
  for v, k in zip(cb.variants, kernels):
    bufs[out_name].zero_()
    try:
      first = timed(k)
    except LaunchError as exc:  # e.g. a launch shape the device rejects: not a candidate
      results.append({'variant': v, 'ms': float('inf'), 'ok': False, 'err': None, 'error': str(exc)})
      continue
    err = float((bufs[out_name] - ref).abs().max()) / scale
    best = first
    if first < slow_ms:  # variants slower than slow_ms are far from the best: one launch suffices
      for _ in range(warmup):
        run(k)
      for _ in range(reps):
        best = min(best, timed(k))
    results.append({'variant': v, 'ms': best, 'ok': err <= check_tol, 'err': err})
  if path:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, 'w') as f:
      json.dump({'chain': cb.spec.key(), 'default': cb.default, 'results': results}, f)
  return results
