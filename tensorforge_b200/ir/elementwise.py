"""Lowering of elementwise statements (`ElementwiseDescr`) into a chain stage.

What the reference's ElementwiseInstruction sets up (backend/instructions/compute/
elementwise.py:29-65) is resolved here at generation time: the index box (n0, n1, ...),
whose sizes come from the tensors' view boxes (optree.py:229-238), and for every tensor
variable the element-relative address of the entry it reads or writes at a point:

    entry = view.bbox.lower + n      address = sum_j (entry_j - origin_j) * stride_j

with origin and strides those of a multilinear operand of the same tensor (the tensor's
box lower corner and column-major strides over its shape; a temporary's own extent).

Points must not interfere, so that every point can run on its own lane: a tensor that
the statements write must be indexed by every index, and every use of it in the stage
must use the same indices and view. Accesses must stay inside the tensor (the shape, a
sparse tensor's pattern box, a temporary's extent); writes go to batched operands and
temporaries only, and never to sparse ones.
"""
from functools import reduce
from typing import Dict, List

from ..common.basic_types import Addressing
from ..common.exceptions import GenerationError
from ..generators import optree as ot


def _prod(xs):
  return reduce(lambda a, b: a * b, xs, 1)


def _colmajor(sizes):
  out, acc = [], 1
  for s in sizes:
    out.append(acc)
    acc *= s
  return out


class EwAccess:
  """How one tensor variable reaches its operand at point n."""

  def __init__(self, op, dims, base, origin, strides):
    self.op = op              # chain Operand
    self.dims = dims          # loop index (0-based) of every tensor dimension
    self.base = base          # absolute entry index at n = 0 (the view's lower corner)
    self.origin = origin
    self.strides = strides

  def key(self):
    return (tuple(self.dims), tuple(self.base))


class EwRef:
  """Operand read by the stage (for the chain-level byte and feature accounting)."""

  def __init__(self, op, target):
    self.op = op
    self.target = target


class EwStage:
  """One `ElementwiseDescr` over the index box `sizes`."""
  kind = 'elementwise'

  def __init__(self, descr, sizes, access, written, read, extents):
    self.descr = descr
    self.statements = descr.oplist
    self.sizes = list(sizes)
    self.n_ranges = [(0, s) for s in sizes]
    self.k_ranges = []
    self.access: Dict[int, EwAccess] = access     # id(variable node) -> access
    self.written = written                        # operands stored to
    self.read = read                              # operands loaded from
    self.extents = extents                        # temporaries defined here -> [(lo, up)]
    self.dest = None
    self.add = False
    self.ops = [EwRef(o, []) for o in read]

  def out_volume(self):
    return _prod(self.sizes)

  def k_volume(self):
    return 1

  def is_matmul(self):
    return False

  def temporaries(self):
    """Distinct TempVar nodes of the statements, in first-appearance order."""
    seen, out = set(), []
    for s in ot.walk_statements(self.statements):
      for root in ot.statement_exprs(s):
        for node in ot.walk_nodes(root):
          if isinstance(node, ot.TempVar) and id(node) not in seen:
            seen.add(id(node))
            out.append(node)
    return out

  def op_count(self):
    """Operation nodes evaluated per point (each loop body counted once)."""
    n = 0
    for s in ot.walk_statements(self.statements):
      for root in ot.statement_exprs(s):
        n += sum(1 for node in ot.walk_nodes(root) if isinstance(node, ot.OpNode))
    return n

  def nz_flops(self):
    return self.op_count() * self.out_volume()

  def dense_flops(self):
    return self.nz_flops()

  def touched_volume(self, o):
    best = 0
    for acc in self.access.values():
      if acc.op is o:
        best = max(best, _prod([self.sizes[d] for d in acc.dims]))
    return best

  def defines_volume(self, o):
    ext = self.extents.get(o.name)
    return _prod([u - l for l, u in ext]) if ext else 0


def _occurrences(statements):
  """(variable node, is_store) in program order: a value before its target, a condition
  before its block."""
  out = []
  for s in ot.walk_statements(statements):
    if isinstance(s, ot.Assignment):
      out += [(n, False) for n in ot.walk_nodes(s.optree) if isinstance(n, (ot.TensorVar, ot.ScalarVar))]
      if isinstance(s.dest, (ot.TensorVar, ot.ScalarVar)):
        out.append((s.dest, True))
      elif not isinstance(s.dest, ot.TempVar):
        raise GenerationError(f'cannot assign to {s.dest}')
    else:
      out += [(n, False) for n in ot.walk_nodes(s.condition) if isinstance(n, (ot.TensorVar, ot.ScalarVar))]
  return out


def lower_elementwise(descr, ops_by_tensor, tmp_ranges) -> EwStage:
  """Resolve one ElementwiseDescr. `tmp_ranges` (id(Operand) -> absolute extent) is read
  for temporaries written earlier and extended with the ones this stage defines."""
  occ = _occurrences(descr.oplist)
  for node, _ in occ:
    if node.tensor is None:
      raise GenerationError('an elementwise variable is not bound to a tensor (assignTensor was not called)')
    rank = node.tensor.bbox.rank()
    if len(node.indices) != rank:
      raise GenerationError(f'{node}: {len(node.indices)} indices for a rank-{rank} tensor')
    if any((not isinstance(i, int)) or i >= 0 for i in node.indices):
      raise GenerationError(f'{node}: elementwise indices are negative (-1 for n0, -2 for n1, ...)')
  ranges = {}
  for s in descr.oplist:
    ranges = s.getRanges(ranges)
  r = len(ranges)
  for i in range(r):
    if -(i + 1) not in ranges:
      raise GenerationError(f'elementwise indices must be n0..n{r - 1} without gaps, got {sorted(ranges)}')
  sizes = [ranges[-(i + 1)][1] for i in range(r)]
  if any(s <= 0 for s in sizes):
    raise GenerationError(f'empty index range in elementwise statements {descr}')

  access: Dict[int, EwAccess] = {}
  written: List = []
  read: List = []
  extents = {}
  for node, store in occ:
    sub = node.tensor
    o = ops_by_tensor[id(sub.tensor)]
    dims = [-i - 1 for i in node.indices]
    base = list(sub.bbox.lower())
    if store:
      if o.kind in ('shared', 'scalar', 'data'):
        raise GenerationError(f'{o.name}: a shared, scalar or compile-time tensor cannot be written')
      if o.sparse:
        raise GenerationError(f'{o.name}: a sparse tensor cannot be written by elementwise statements')
      if set(dims) != set(range(r)):
        raise GenerationError(f'{o.name} is written but not indexed by every index n0..n{r - 1}: '
                              'points would write the same entry')
    if o.kind == 'tmp':
      rng = tmp_ranges.get(id(o))
      if rng is None:
        if not store:
          raise GenerationError(f'temporary {o.name} is read before it is written')
        if len(set(dims)) != len(dims):
          raise GenerationError(f'temporary {o.name} is defined through a repeated index')
        rng = [(b, b + sizes[d]) for b, d in zip(base, dims)]
        tmp_ranges[id(o)] = rng
        extents[o.name] = rng
      origin = [l for l, _ in rng]
      strides = _colmajor([u - l for l, u in rng])
      limits = [(l, u) for l, u in rng]
      for (lo, up), b, d in zip(limits, base, dims):
        if b < lo or b + sizes[d] > up:
          raise GenerationError(f'{node} reaches outside the extent of temporary {o.name}')
    elif o.kind in ('batched', 'shared'):
      origin = list(o.bbox.lower())
      extent = list(o.tensor.spp.indexmask.shape) if o.sparse else list(o.shape)
      strides = _colmajor(extent)
      for j, (b, d) in enumerate(zip(base, dims)):
        if b - origin[j] < 0 or b - origin[j] + sizes[d] > extent[j]:
          raise GenerationError(f'{node} reaches outside {o.name} (dimension {j})')
    else:  # scalar argument or compile-time values (read at the absolute entry)
      origin = [0] * len(dims)
      strides = [0] * len(dims)
      for j, (b, d) in enumerate(zip(base, dims)):
        if b < 0 or b + sizes[d] > o.shape[j]:
          raise GenerationError(f'{node} reaches outside {o.name} (dimension {j})')
    acc = EwAccess(o, dims, base, origin, strides)
    access[id(node)] = acc
    if store and all(x is not o for x in written):
      written.append(o)
    if not store and all(x is not o for x in read):
      read.append(o)
  # a written operand is used the same way everywhere in the stage
  for o in written:
    keys = {acc.key() for acc in access.values() if acc.op is o}
    if len(keys) != 1:
      raise GenerationError(f'{o.name} is written and used with different indices or views in one '
                            'elementwise stage')
  for acc in access.values():
    if acc.op.kind == 'scalar' and acc.op.addressing != Addressing.SCALAR:
      raise GenerationError(f'{acc.op.name}: unsupported scalar operand')
  return EwStage(descr, sizes, access, written, read, extents)
