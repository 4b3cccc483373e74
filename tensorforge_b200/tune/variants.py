"""Tunable variants of a chain and the cost model's 32-dim feature vectors."""
import math

from ..plan import SMEM_LIMIT
from ..plan.chains import match_left_chain

GENERIC_G = (4, 8, 16, 32, 64, 128, 256)
GENERIC_E = (1, 2, 4, 8, 16)
COLPROG = [dict(threads=t, a_source=a) for t in (128, 256) for a in ("const", "smem")]
# points each lane evaluates per pass in elementwise stages (generic generator)
POINTS_PER_LANE = (1, 2, 4, 8)
# tensor-core (TF32x3) variants: operand form U with the warp-specialised (3) or one-pass (2)
# producer pipeline, operand form B with one or two B buffers
TCSPLIT = [{'strategy': 'tcsplit', 'form': 'u', 'pipe': 3}, {'strategy': 'tcsplit', 'form': 'u', 'pipe': 2},
           {'strategy': 'tcsplit', 'form': 'b', 'bbuf': 1}, {'strategy': 'tcsplit', 'form': 'b', 'bbuf': 2}]
NFEAT = 32
TUNE_COLPROG_MAX_FMAS = 2048


def tensor_core_space(chain, precision='tf32x3'):
  """Tensor-core variants that the planner realises for `chain` (distinct plans only)."""
  from ..plan.chains import tcsplit_plan
  shape = match_left_chain(chain)
  if shape is None:
    return []
  out, seen = [], set()
  for v in TCSPLIT:
    p = tcsplit_plan(chain, shape, precision, v)
    if p is None or p.key() in seen:
      continue
    seen.add(p.key())
    out.append(dict(v))
  return out


def variant_space(chain, fp_size=4, precision='plain', model_only=False):
  """Variant dicts (Options.variant) that apply to `chain`.

  precision 'tf32x3': the tensor-core variants (timed by the exhaustive tuner). For plain
  chains with elementwise stages the generic variants also vary the points per lane,
  except with `model_only` (the cost model was trained on the default of 4)."""
  from ..codegen.generic import smem_layout
  if precision == 'tf32x3':
    return tensor_core_space(chain, precision)
  out = []
  shared, per_elem = smem_layout(chain)
  ppl = (None,) if (model_only or not chain.has_elementwise()) else POINTS_PER_LANE
  for g in GENERIC_G:
    for e in GENERIC_E:
      if g * e > 1024 or g * e < 32:
        continue
      if (shared + per_elem * e) * fp_size > SMEM_LIMIT:
        continue
      for u in ppl:
        v = {'strategy': 'generic', 'threads_per_element': g, 'elements_per_block': e}
        if u is not None:
          v['points_per_lane'] = u
        out.append(v)
  shape = match_left_chain(chain)
  if shape is not None and shape.M <= 128 and shape.N <= 128:
    # tuning builds every variant; column programs with large A cost ptxas close to a
    # minute each, so only the planner's own column program is measured for those
    if sum(t.A.storage_size() for t in shape.terms) <= TUNE_COLPROG_MAX_FMAS:
      for v in COLPROG:
        if shape.N <= v['threads']:
          out.append(dict(strategy='colprog', **v))
  return out


def _l2(x):
  return math.log2(max(1.0, float(x)))


def _stage_density(stage):
  """Density of the stage's stored (non-temporary) operands: the sparsest one's."""
  d = [r.op.tensor.density() for r in stage.ops if r.op.kind != 'tmp' and r.op.sparse]
  return min(d) if d else 1.0


def chain_features(chain, batch):
  """20 features of the lowered chain and its batch size (up to 4 stages described)."""
  st = chain.stages
  f = [len(st) / 4.0]
  for i in range(4):
    if i < len(st):
      s = st[i]
      rows = s.n_ranges[0][1] - s.n_ranges[0][0] if s.n_ranges else 1
      cols = s.n_ranges[1][1] - s.n_ranges[1][0] if len(s.n_ranges) > 1 else 1
      f += [_l2(rows) / 7.0, _l2(cols) / 7.0, _l2(s.k_volume()) / 7.0, _stage_density(s)]
    else:
      f += [0.0, 0.0, 0.0, 0.0]
  f.append(math.log10(max(1, batch)) / 6.0)
  f.append(math.log10(max(1.0, chain.nz_flops_per_element())) / 7.0)
  f.append(math.log10(max(1.0, chain.bytes_per_element())) / 6.0)
  return f


def variant_features(chain, variant, fp_size=4):
  """12 features of the variant (strategy, launch shape, shared memory).

  `variant` holds the parameters the planner actually applied (the plan's params plus
  'strategy'), not the requested ones: a requested constant-memory A that does not fit
  falls back to shared memory, for example.
  """
  from ..codegen.generic import smem_layout
  shared, per_elem = smem_layout(chain)
  if variant['strategy'] == 'generic':
    g, e = variant['threads_per_element'], variant['elements_per_block']
    smem = (shared + per_elem * e) * fp_size
    ppl = variant.get('points_per_lane', 4) if chain.has_elementwise() else 0
    return [1.0, 0.0, _l2(g) / 6.0, _l2(e) / 4.0, g * e / 1024.0, 0.0, 0.0, smem / SMEM_LIMIT,
            math.log10(max(1, per_elem * fp_size)) / 5.0, 0.0, 0.0, ppl / 8.0 if ppl != 4 else 0.0]
  t = variant['threads']
  shape = match_left_chain(chain)
  te = max(1, t // shape.N)
  return [0.0, 1.0, 0.0, _l2(te) / 6.0, t / 1024.0, 1.0 if variant['a_source'] == 'const' else 0.0,
          te * shape.N / t, 0.0, 0.0, shape.M / 128.0, len(shape.terms) / 4.0, 0.0]


def features(chain, variant, batch):
  """The cost model's input for running `variant` of `chain` on `batch` elements."""
  memo = chain.__dict__.setdefault('_tune_features', {})
  if batch not in memo:  # the chain part is shared by all variants (and costs a nonzero count)
    memo[batch] = chain_features(chain, batch)
  f = memo[batch] + variant_features(chain, variant)
  assert len(f) == NFEAT, len(f)
  return f


def effective_variant(plan):
  """The variant dict a plan realises (its strategy and applied parameters)."""
  return dict(strategy=plan.strategy, **plan.params)


def space_signature():
  """Short hash of the variant space: tuning results are only comparable within one space."""
  import hashlib
  key = repr((GENERIC_G, GENERIC_E, COLPROG, TUNE_COLPROG_MAX_FMAS, NFEAT))  # the timed plain space
  return hashlib.sha1(key.encode()).hexdigest()[:8]
