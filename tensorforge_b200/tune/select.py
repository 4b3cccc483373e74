"""Variant selection at generation time: `Options(tuner='model')` and `tuner='exhaustive'`.

'model'       ranks every applicable variant with the trained cost model (weights shipped
              in model_b200.npz, trained on B200 timings) and takes the best predicted
              one. The network runs on the GPU through the native MLP kernels
              (tfb_mlp_forward) when a CUDA device is present; generation on a machine
              without one evaluates the same network on the host.
'exhaustive'  builds every variant and times it on the current GPU (CUDA events, best of
              3) with synthetic inputs of `batch` elements, and takes the fastest.

'model' chooses among the plain-precision variants it was trained on (generic lane
groups and elements per CTA, column programs). 'exhaustive' also times the points per
lane of elementwise stages and, for precision 'tf32x3', the tensor-core variants
(operand forms U and B, producer pipelines). Launchers are generic in numElements, so
the batch the choice is made for is a parameter (default 100,000).
"""
import os

import numpy as np

from .variants import variant_space, features

DEFAULT_BATCH = 100_000
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'model_b200.npz')
_model = None


def _load_model():
  global _model
  if _model is None:
    if not os.path.exists(MODEL_PATH):
      raise FileNotFoundError(f'cost model weights missing: {MODEL_PATH}')
    z = np.load(MODEL_PATH)
    _model = (z['params'], z['mean'], z['std'])
  return _model


_gpu_model = None
last_inference = None   # 'gpu' or 'host': where the latest model_choice ran the network


def _device_model():
  """The shipped weights in a CostModel on the GPU (native MLP kernels), or None when no
  CUDA device (or no native runtime library) is available."""
  global _gpu_model
  if _gpu_model is None:
    try:
      import torch
      if not torch.cuda.is_available():
        return None
      from .cost_model import CostModel
      m = CostModel()
      m.load(MODEL_PATH)
      _gpu_model = m
    except (ImportError, OSError, RuntimeError):
      return None
  return _gpu_model


def predict(feats):
  """Predicted log-runtimes of feature rows: on the GPU when possible, else on the host."""
  global last_inference
  m = _device_model()
  if m is not None:
    last_inference = 'gpu'
    return m.predict(feats)
  from .cost_model import host_predict
  params, mean, std = _load_model()
  last_inference = 'host'
  return host_predict(params, mean, std, feats)


def model_choice(chain, fp_size=4, batch=DEFAULT_BATCH):
  """Variant dict with the lowest predicted runtime, or None if there is no choice."""
  cands = variant_space(chain, fp_size, model_only=True)
  if len(cands) < 2:
    return None
  pred = predict([features(chain, v, batch) for v in cands])
  return cands[int(np.argmin(pred))]


def exhaustive_choice(descr_list, context, batch=DEFAULT_BATCH, reps=3):
  """Build and time every variant of `descr_list` on the current GPU; the fastest wins."""
  import torch
  from ..common.context import Context, Options
  from ..generators.generator import Generator
  from ..runtime.kernel import CompiledKernel
  opts = context.get_user_options()

  def gen(variant):
    o = Options(opts.exact_contraction_length, opts.align_shr_mem, opts.enable_sync_block_opt,
                opts.precision, 'heuristic', variant)
    g = Generator(descr_list, Context(context.arch, context.backend, context.fp_type, o))
    g.generate()
    return g

  base = gen(None)
  cands = variant_space(base.get_chain(), context.fp_type.size(), opts.precision)
  if len(cands) < 2:
    return None
  dtype = torch.float64 if context.fp_type.size() == 8 else torch.float32
  bufs = {}
  for t, _ in base.abi_symbols():
    if t.addressing.name == 'SCALAR':
      continue
    if t.addressing.name == 'PTR_BASED':
      return None  # pointer arrays would need per-element buffers: keep the heuristic plan
    size = t.spp.count_nz() if t.addressing.name == 'NONE' else batch * t.get_real_volume()
    bufs[t.name] = torch.rand(max(1, size), device='cuda', dtype=dtype)
  scalars = {t.name: 1.0 for t, _ in base.abi_symbols() if t.addressing.name == 'SCALAR'}
  stream = torch.cuda.current_stream()
  best, best_ms = None, float('inf')
  for v in cands:
    k = CompiledKernel(gen(v))
    kw = dict(bufs, **scalars)
    k(numElements=batch, **kw)
    for _ in range(reps):
      s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      s.record(stream)
      k(numElements=batch, **kw)
      e.record(stream)
      e.synchronize()
      ms = s.elapsed_time(e)
      if ms < best_ms:
        best, best_ms = v, ms
  return best
