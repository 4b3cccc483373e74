"""Shared-left GEMM chains: recognition and plans for the fast generators.

A chain qualifies when it computes, for every batch element e,

    out_e  (+)=  sum_t  A_t * B_{e,t} * R_{e,t}

with A_t shared across the batch (Addressing.NONE, dense or sparse), B_{e,t} batched and
dense, R_{e,t} batched or shared (dense or sparse) or absent, written in the
reference's descriptor form (tensorforge/generators/descriptions.py:14-27):

    T_t  =  A_t x B_t            (temporary, targets [[0,-1],[-1,1]])
    out (+)= T_t x R_t           (targets [[0,-1],[-1,1]], add for t > 0)

or a single `out (+)= A x B`. All operands must span their full shape (bounding box =
shape) so that columns are contiguous. This is the shape of BASELINE configs 0-3
(benchmarks/fused/programs/s3time.cf) and of SeisSol's volume/local kernels.
"""
from dataclasses import dataclass, field
from typing import List, Optional

from ..common.basic_types import DataFlowDirection
from . import Plan, SMEM_LIMIT


@dataclass
class Term:
  A: object          # Operand (shared)
  B: object          # Operand (batched, dense)
  R: Optional[object]  # Operand (batched/shared) or None
  K: int
  P: int


@dataclass
class LeftChain:
  terms: List[Term]
  out: object
  M: int
  N: int
  accumulate: bool   # out_e += ... (previous value read once)
  epilogue: list = field(default_factory=list)   # elementwise stages on the output, per entry


def _full(op):
  t = op.tensor
  return list(t.bbox.lower()) == [0] * len(t.shape) and list(t.bbox.upper()) == list(t.shape)


def _full_ref(stage, ref):
  box = [stage.n_ranges[x] if x >= 0 else stage.k_ranges[-x - 1] for x in ref.target]
  return [l for l, _ in box] == [0] * len(box) and [u for _, u in box] == list(ref.op.shape)


def _is_elementwise(stage):
  return getattr(stage, 'kind', '') == 'elementwise'


def _epilogue_ok(tail, shape):
  """Elementwise stages that can run on the output's registers: over the output's whole
  M x N box, writing the output only, reading the output, scalars and batched dense M x N
  tensors at the same entry (n0 = row, n1 = column)."""
  out = shape.out
  for s in tail:
    if s.sizes != [shape.M, shape.N] or any(o is not out for o in s.written):
      return False
    for acc in s.access.values():
      o = acc.op
      if o.kind in ('scalar', 'data') and not acc.dims:
        continue
      if o.kind != 'batched' or o.sparse or not _full(o) or list(o.shape) != [shape.M, shape.N]:
        return False
      if acc.dims != [0, 1] or acc.base != [0, 0]:
        return False
  return True


def match_left_chain(chain) -> Optional[LeftChain]:
  """The chain's shared-left form, with trailing elementwise stages as an epilogue."""
  st = chain.stages
  k = next((i for i, s in enumerate(st) if _is_elementwise(s)), len(st))
  tail = st[k:]
  st = st[:k]
  if not st or not all(_is_elementwise(s) for s in tail):
    return None
  for s in st:
    if not s.is_matmul():
      return None
    for r in s.ops:
      if r.op.kind == 'tmp':
        continue
      if r.op.kind not in ('shared', 'batched') or not _full(r.op) or not _full_ref(s, r):
        return None
  out = None
  terms = []
  i = 0
  accumulate = False
  while i < len(st):
    s = st[i]
    if s.dest.kind == 'tmp':
      if i + 1 >= len(st):
        return None
      s2 = st[i + 1]
      a, b = s.ops
      t, r = s2.ops
      if t.op is not s.dest or s2.dest.kind != 'batched' or s.add:
        return None
      if r.op.kind == 'tmp':
        return None
      if a.op.kind != 'shared' or b.op.kind != 'batched' or b.op.sparse:
        return None
      # the temporary must not be used anywhere else
      if sum(1 for x in st for y in x.ops if y.op is s.dest) != 1:
        return None
      dest = s2.dest
      term = Term(a.op, b.op, r.op, a.op.shape[1], b.op.shape[1])
      add = s2.add
      i += 2
    else:
      if s.dest.kind != 'batched':
        return None
      a, b = s.ops
      if a.op.kind != 'shared' or b.op.kind != 'batched' or b.op.sparse:
        return None
      dest = s.dest
      term = Term(a.op, b.op, None, a.op.shape[1], b.op.shape[1])
      add = s.add
      i += 1
    if dest.sparse or not _full(dest):
      return None
    if out is None:
      out = dest
      accumulate = add
    elif dest is not out or not add:
      return None
    terms.append(term)
  M, N = out.shape
  for t in terms:
    if t.A.shape[0] != M or t.B.shape[0] != t.K:
      return None
    if t.R is None and t.P != N:
      return None
    if t.R is not None and (t.R.shape[0] != t.P or t.R.shape[1] != N):
      return None
    if t.B is out or t.A is out or t.R is out:
      return None
  shape = LeftChain(terms, out, M, N, accumulate)
  if tail:
    if not _epilogue_ok(tail, shape):
      return None
    shape.epilogue = list(tail)
  return shape


def a_values(term):
  """Consumption order of A_t's nonzeros: column l outer, row i inner.

  Returns [(l, [(i, storage position), ...]), ...] for l = 0..K-1.
  """
  A = term.A
  M, K = A.shape
  if A.sparse:
    look = A.sparse_lookup()
    cols = []
    for l in range(K):
      rows = [(i, look[(i, l)]) for i in range(M) if (i, l) in look]
      cols.append((l, rows))
    return cols
  return [(l, [(i, l * M + i) for i in range(M)]) for l in range(K)]


def r_slots(term):
  """Per output column j: [(m, storage position)] of R_t's nonzeros in column j."""
  R = term.R
  P, N = R.shape
  if R.sparse:
    look = R.sparse_lookup()
    return [[(m, look[(m, j)]) for m in range(P) if (m, j) in look] for j in range(N)]
  return [[(m, j * P + m) for m in range(P)] for j in range(N)]


# Column programs unroll one FMA per nonzero of every A_t into straight-line code. Above
# this many ptxas time grows past a minute per kernel, so such chains go to the generic
# generator. Measured on B200 (84x84 A at 45 %, three terms, 9,533 FMAs per column, 26 s of
# ptxas, 226 registers, no spills): 2.13e7 against 2.30e6 el/s for the generic kernel with 27
# quantities and 8.25e7 against 1.04e7 with 9, so the larger code still pays many times over.
COLPROG_MAX_FMAS = 16384
# A 128-thread column program whose shared memory leaves room for only one CTA per SM runs
# with 256 threads instead when that keeps the prefetch stage (same registers per thread,
# twice the warps per SM; 2.0x and 1.9x faster on the two 84-basis chains above).
COLPROG_SMEM_PER_SM = 228 * 1024
# A values as constant-bank FMA operands stay in the immediate-constant cache up to roughly
# this many values. Measured on B200: constant A is fastest for most random chains with at
# most 2,048 values and for the dense 56x56 GEMM (3,136 values: 2.54e8 vs 2.32e8 el/s);
# the order-6 chain (4,253 values over three terms) runs 1.24x faster from shared memory.
COLPROG_CONST_A = 4096


# Variant 'mixed' (not a default): the leading terms whose A values fit this budget stay
# constant-bank FMA operands and the rest move to shared memory. With an odd U pitch it
# brings the order-6 chain's CTA to 72 KB of shared memory and 167 registers, three CTAs per
# SM instead of two -- measured slower (2.61e8 against 2.71e8 el/s), as were the other
# three-CTA forms (2.49e8-2.65e8).
COLPROG_CONST_MIXED = 2048


def colprog_plan(chain, shape: LeftChain, fp_size, variant):
  if 'threads' in variant:
    return _colprog_plan(chain, shape, fp_size, variant, variant['threads'])
  p = _colprog_plan(chain, shape, fp_size, variant, 128)
  if p is not None and 2 * (p.smem_bytes + 1024) > COLPROG_SMEM_PER_SM:
    wide = _colprog_plan(chain, shape, fp_size, variant, 256)
    # only where the wider tile keeps the prefetch stage (measured only in that form)
    if wide is not None and wide.params['prefetch'] >= p.params['prefetch']:
      return wide
  return p


def _colprog_plan(chain, shape: LeftChain, fp_size, variant, threads):
  from ..codegen.colprog import tile_elements
  chunk = variant.get('chunk', 16)
  sizes = [t.A.storage_size() for t in shape.terms]
  a_total = sum(sizes)
  if 'a_source' in variant:
    a_source = variant['a_source']
  elif a_total <= COLPROG_CONST_A:
    a_source = 'const'
  else:
    a_source = 'smem'
  const_terms = int(variant.get('const_terms', 0))
  if a_source == 'mixed' and 'const_terms' not in variant:
    acc = 0
    for n in sizes:
      if acc + n > COLPROG_CONST_MIXED:
        break
      acc += n
      const_terms += 1
    if const_terms == 0:
      a_source = 'smem'
  vec = 4 if fp_size == 4 else 2
  chunk = max(vec, (chunk + vec - 1) // vec * vec)
  if shape.M > 128 or shape.N > threads:
    return None
  if a_total > COLPROG_MAX_FMAS and variant.get('strategy') != 'colprog':
    return None
  cols = int(variant.get('cols', 1))
  rsplit = int(variant.get('rsplit', 1))
  if rsplit > 1 and (shape.epilogue or threads % rsplit or shape.N > threads // rsplit):
    rsplit = 1   # the elementwise epilogue needs whole columns in one thread
  te = tile_elements(shape, threads // rsplit, cols)
  kmax = max(t.K for t in shape.terms)
  upitch = variant.get('upitch', 'odd' if a_source == 'mixed' else 'vec')
  pitch = (kmax | 1) if upitch == 'odd' else (kmax + vec - 1) // vec * vec + vec
  if a_source == 'const' and a_total * fp_size > 48 * 1024:
    a_source = 'smem'
  n_const = {'const': len(sizes), 'smem': 0}.get(a_source, const_terms)
  a_smem_vals = sum(sizes[n_const:])
  prefetch = int(variant.get('prefetch', 1))
  smem = max(te * shape.N * pitch, te * shape.N * shape.M) * fp_size
  r_staged = sum(te * ((t.R.storage_size() + vec - 1) // vec * vec) for t in shape.terms
                 if t.R is not None and t.R.kind == 'batched') * fp_size
  if a_smem_vals:
    smem += (a_smem_vals + vec) * fp_size
  stage = sum(te * ((op.storage_size() if op.sparse else op.element_volume()) + vec - 1) // vec * vec
              for op in {id(o): o for t in shape.terms for o in (t.B, t.R)
                         if o is not None and o.kind == 'batched'}.values()) * fp_size
  if not prefetch or smem + stage > SMEM_LIMIT:
    prefetch = 0
    smem += r_staged
  else:
    smem += stage
  if smem > SMEM_LIMIT:
    return None
  # __launch_bounds__(128, 2) measured 4-5 % faster on the order-6 chain at every chunk size
  # (2.60e8 -> 2.70e8 el/s at chunk 16); 256-thread CTAs gain nothing from it
  default_mb = 2 if threads == 128 and rsplit == 1 else 0
  params = {'threads': threads, 'chunk': chunk, 'min_blocks': variant.get('min_blocks', default_mb),
            'a_source': a_source, 'prefetch': prefetch}
  if a_source == 'mixed':
    params['const_terms'] = n_const
  if upitch != 'vec':
    params['upitch'] = upitch
  if cols != 1:
    params['cols'] = cols
  if rsplit != 1:
    params['rsplit'] = rsplit
  return Plan('colprog', params,
              smem, threads, note=f'M={shape.M} N={shape.N} terms={len(shape.terms)} tile={te}')


def tcsplit_plan(chain, shape, precision, variant):
  if shape.epilogue:  # elementwise epilogues run on the column programs only
    return None
  from ..codegen import tcsplit
  return tcsplit.plan(chain, shape, precision, variant)


def dmma_plan(chain, shape, variant):
  if shape.epilogue:
    return None
  from ..codegen import dmma
  return dmma.plan(chain, shape, variant, SMEM_LIMIT)
