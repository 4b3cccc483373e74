"""Chain IR: a lowered, fully resolved form of a descriptor list.

The frontend descriptors (`MultilinearDescr`) are turned into `Stage`s over `Operand`s.
Everything the code generators need is resolved here at generation time: the index
ranges of every output and contracted index (bounding-box intersections, as in
tensorforge/backend/instructions/compute/multilinear.py:58-96), the element-relative
address of every operand entry (ptr_manip.py:19-65, symbol.py:304-330, load.py:76-137),
and the nonzero list of every sparse operand (spp.py, symbol.py:340-401).
"""
from dataclasses import dataclass, field
from functools import reduce
from typing import Dict, List, Optional, Tuple
import math

from ..common.basic_types import Addressing, DataFlowDirection, FloatingPointType
from ..common.exceptions import GenerationError
from ..common.matrix.tensor import Tensor, SubTensor


def _prod(xs):
  return reduce(lambda a, b: a * b, xs, 1)


@dataclass
class Operand:
  """One tensor of the chain.

  kind: 'batched' (STRIDED / PTR_BASED, one copy per element), 'shared' (NONE),
        'scalar' (SCALAR, by value), 'data' (compile-time values, not in the ABI),
        'tmp' (intermediate, lives on chip only).
  """
  name: str
  tensor: Tensor
  kind: str
  abi_index: int = -1          # position among ABI symbols (m-order), -1 if not in the ABI

  @property
  def addressing(self):
    return self.tensor.addressing

  @property
  def shape(self):
    return self.tensor.shape

  @property
  def bbox(self):
    return self.tensor.bbox

  @property
  def sparse(self):
    return self.kind in ('batched', 'shared') and self.tensor.is_sparse_storage()

  @property
  def is_const(self):
    return self.tensor.direction == DataFlowDirection.SOURCE

  def element_volume(self):
    """Elements between consecutive batch copies of a STRIDED operand (ptr_manip.py:37-45)."""
    return self.tensor.get_real_volume()

  def storage_size(self):
    """Number of values one batch copy occupies (dense: strided span; sparse: nnz)."""
    if self.sparse:
      return max([p for _, p in self.tensor.spp.nonzeros()] + [-1]) + 1
    return self.tensor.get_real_volume()

  def nonzeros(self):
    """(absolute index, storage position) of every stored entry of a sparse operand."""
    lo = self.tensor.bbox.lower()
    return [(tuple(r + l for r, l in zip(rel, lo)), pos) for rel, pos in self.tensor.spp.nonzeros()]

  def sparse_lookup(self) -> Dict[Tuple[int, ...], int]:
    """Absolute index -> storage position of a sparse operand.

    Entries outside the pattern's index mask are absent (value 0), matching
    `ListSPP.linear_index` returning None (spp.py:102-107).
    """
    out = self.__dict__.get('_lookup')
    if out is None:  # built once: the pattern of an operand never changes after lowering
      out = self.__dict__['_lookup'] = {idx: pos for idx, pos in self.nonzeros()}
    return out


@dataclass
class OpRef:
  """Operand `op` used in a stage, with the dimension -> index mapping `target`."""
  op: Operand
  view: object                 # BoundingBox of the SubTensor view
  target: List[int]
  strides: List[int] = field(default_factory=list)   # element-relative address = sum (idx-origin)*stride
  origin: List[int] = field(default_factory=list)


@dataclass
class Stage:
  dest: Operand
  dest_view: object
  ops: List[OpRef]
  add: bool
  n_ranges: List[Tuple[int, int]]
  k_ranges: List[Tuple[int, int]]
  dest_strides: List[int] = field(default_factory=list)
  dest_origin: List[int] = field(default_factory=list)
  descr: object = None

  def out_volume(self):
    return _prod([u - l for l, u in self.n_ranges])

  def k_volume(self):
    return _prod([u - l for l, u in self.k_ranges])

  def is_matmul(self):
    """True for a plain 2-operand product dest[i,j] = sum_k A[i,k] B[k,j] (no scalars)."""
    if len(self.ops) != 2 or len(self.n_ranges) != 2 or len(self.k_ranges) != 1:
      return False
    return self.ops[0].target == [0, -1] and self.ops[1].target == [-1, 1]

  def nz_flops(self):
    """Multiply-adds counted over nonzero operand entries only, times 2."""
    return 2 * count_products(self)

  def dense_flops(self):
    return 2 * self.out_volume() * self.k_volume()

  def touched_volume(self, o):
    best = self.out_volume() if self.dest is o else 0
    for r in self.ops:
      if r.op is o:
        best = max(best, _prod([u - l for l, u in _op_box(self, r)]))
    return best

  def defines_volume(self, o):
    return self.out_volume() if self.dest is o else 0


def stored_targets(descr):
  """Targets per operand in the operand's stored dimension order.

  `target[i][d]` names the index of dimension d of operand i *as permuted by*
  `permute[i]` (view dimension d is stored dimension permute[i][d]), which is how
  GemmDescr expresses transposes (descriptions.py:126-149: trans_a -> permute [1, 0] with
  target [0, -1]). The reference itself stops with NameError for any non-identity
  permute, so this is the intent of its interface rather than observed behaviour.
  """
  out = []
  for i, tgt in enumerate(descr.target):
    perm = descr.permute[i] if descr.permute is not None and i < len(descr.permute) else None
    if not perm or len(perm) != len(tgt) or sorted(perm) != list(range(len(tgt))):
      out.append(list(tgt))
      continue
    eff = [0] * len(tgt)
    for view_dim, stored_dim in enumerate(perm):
      eff[stored_dim] = tgt[view_dim]
    out.append(eff)
  return out


def count_products(stage: Stage) -> int:
  """Number of nonzero scalar products of one stage (used for nz-FLOP rooflines)."""
  if stage.is_matmul():
    a, b = stage.ops
    (i0, i1), (j0, j1) = stage.n_ranges
    k0, k1 = stage.k_ranges[0]
    rows_per_k = {}
    cols_per_k = {}
    for k in range(k0, k1):
      rows_per_k[k] = sum(1 for i in range(i0, i1) if entry_nonzero(a, (i, k)))
      cols_per_k[k] = sum(1 for j in range(j0, j1) if entry_nonzero(b, (k, j)))
    return sum(rows_per_k[k] * cols_per_k[k] for k in range(k0, k1))
  return stage.out_volume() * stage.k_volume()


def entry_nonzero(ref: OpRef, idx) -> bool:
  op = ref.op
  if op.kind == 'tmp' or not op.sparse:
    return True
  return tuple(idx) in op.sparse_lookup()


@dataclass
class Chain:
  operands: List[Operand]          # ABI symbols, m-order
  tmps: List[Operand]
  stages: List[Stage]
  fp: FloatingPointType

  def batched(self):
    return [o for o in self.operands if o.kind == 'batched']

  def shared(self):
    return [o for o in self.operands if o.kind == 'shared']

  def abi_symbols(self):
    return [o for o in self.operands if o.kind in ('batched', 'shared', 'scalar')]

  def sinks(self):
    return [o for o in self.operands if o.kind == 'batched' and o.tensor.direction != DataFlowDirection.SOURCE]

  def nz_flops_per_element(self):
    return sum(s.nz_flops() for s in self.stages)

  def dense_flops_per_element(self):
    return sum(s.dense_flops() for s in self.stages)

  def has_elementwise(self):
    return any(getattr(s, 'kind', '') == 'elementwise' for s in self.stages)

  def bytes_per_element(self):
    """Algorithmic HBM bytes per element: every batched input read once, every output
    written once (read too if it is accumulated into), shared operands excluded."""
    size = self.fp.size()
    total = 0
    for o in self.batched():
      d = o.tensor.direction
      vol = o.storage_size() if o.sparse else _touched_volume(self, o)
      if d == DataFlowDirection.SOURCE:
        total += vol * size
      else:  # written (and possibly read back): read from memory only before the first overwrite
        total += vol * size * (2 if _reads_dest(self, o) else 1)
      if o.addressing == Addressing.PTR_BASED:
        total += 8
    return total


def _touched_volume(chain, o):
  best = max([s.touched_volume(o) for s in chain.stages] + [0])
  return best if best > 0 else o.tensor.get_actual_volume()


def _reads_dest(chain, o):
  """True when the chain reads o's previous contents from memory: a read, or an
  accumulating write, before the first plain overwrite (later reads see the chain's own
  result, not HBM data the algorithm has to move)."""
  for s in chain.stages:
    if any(r.op is o for r in s.ops):
      return True
    written = any(x is o for x in s.written) if getattr(s, 'kind', '') == 'elementwise' else (s.dest is o)
    if written:
      return bool(s.add)
  return False


def _op_box(stage, ref):
  box = []
  for t in ref.target:
    box.append(stage.n_ranges[t] if t >= 0 else stage.k_ranges[-t - 1])
  return box


def _colmajor_strides(sizes):
  strides, acc = [], 1
  for s in sizes:
    strides.append(acc)
    acc *= s
  return strides


def lower(descr_list, matrix_list, global_symbols, fp: FloatingPointType) -> Chain:
  """Lower named descriptors into a Chain.

  `matrix_list` is every tensor in first-appearance order (already named m*/t*),
  `global_symbols` the ABI symbols as (tensor, stype) in m-order.
  """
  ops_by_tensor: Dict[int, Operand] = {}
  operands: List[Operand] = []
  tmps: List[Operand] = []
  abi_i = 0
  for tensor, stype in global_symbols:
    if stype == 'data':
      kind = 'data'
      if tensor.addressing not in (Addressing.SCALAR,) and tensor.data is None:
        kind = 'batched'
    elif stype == 'scalar':
      kind = 'scalar'
    elif tensor.addressing == Addressing.NONE:
      kind = 'shared'
    else:
      kind = 'batched'
    o = Operand(tensor.name, tensor, kind, abi_i if kind in ('batched', 'shared', 'scalar') else -1)
    if kind in ('batched', 'shared', 'scalar'):
      abi_i += 1
    ops_by_tensor[id(tensor)] = o
    operands.append(o)
  for tensor in matrix_list:
    if tensor.is_tmp and id(tensor) not in ops_by_tensor:
      o = Operand(tensor.name, tensor, 'tmp')
      ops_by_tensor[id(tensor)] = o
      tmps.append(o)

  stages = []
  tmp_ranges: Dict[int, List[Tuple[int, int]]] = {}
  for d in descr_list:
    if hasattr(d, 'oplist'):
      from .elementwise import lower_elementwise
      stages.append(lower_elementwise(d, ops_by_tensor, tmp_ranges))
      continue
    refs = []
    nr: Dict[int, Tuple[int, int]] = {}
    kr: Dict[int, Tuple[int, int]] = {}
    for sub, tgt in zip(d.ops, stored_targets(d)):
      o = ops_by_tensor[id(sub.tensor)]
      refs.append(OpRef(o, sub.bbox, list(tgt)))
      for j, t in enumerate(tgt):
        lo, up = sub.bbox.lower()[j], sub.bbox.upper()[j]
        table = nr if t >= 0 else kr
        key = t if t >= 0 else -t - 1
        if key in table:
          a, b = table[key]
          table[key] = (max(a, lo), min(b, up))
        else:
          table[key] = (lo, up)
    rank = (max(nr.keys()) + 1) if nr else 0
    for t in range(rank):
      if t not in nr:
        raise GenerationError(f'output index n{t} is not produced by any operand of {d}')
    for k in range(len(kr)):
      if k not in kr:
        raise GenerationError(f'contraction indices of {d} are not contiguous')
    n_ranges = [nr[t] for t in range(rank)]
    k_ranges = [kr[k] for k in range(len(kr))]
    for r in n_ranges + k_ranges:
      if r[1] < r[0]:
        raise GenerationError(f'empty index range in {d}')
    dest = ops_by_tensor[id(d.dest.tensor)]
    if dest.kind in ('shared', 'scalar', 'data'):
      if dest.kind == 'shared':
        raise GenerationError('a shared (Addressing.NONE) tensor cannot be written')
      raise GenerationError('a scalar or compile-time tensor cannot be written')
    if len(n_ranges) != len(dest.shape) and dest.kind != 'tmp':
      raise GenerationError(f'result rank {len(n_ranges)} does not match {dest}')
    if dest.kind != 'tmp':
      # the result is stored relative to the destination box's lower corner: every stored
      # index must stay inside the destination's shape (else it would land in another
      # element's data or past the buffer)
      for t, (lo, up) in enumerate(n_ranges):
        base = d.dest.bbox.lower()[t]
        if lo - base < 0 or up - base > dest.shape[t]:
          raise GenerationError(f'result index range n{t} [{lo}, {up}) of {d} does not fit the '
                                f'destination (box from {base}, extent {dest.shape[t]})')
    st = Stage(dest, d.dest.bbox, refs, bool(d.add), n_ranges, k_ranges, descr=d)
    # the reference reads a non-permuted, lead-less dense operand through a compact copy of
    # its bounding box (load.py:76-137); both layouts coincide when the box covers the shape.
    for idx_op, ref in enumerate(st.ops):
      o = ref.op
      dsc_perm = d.permute[idx_op] if idx_op < len(d.permute) else list(range(len(ref.target)))
      identity = list(dsc_perm) == list(range(len(ref.target)))
      if o.kind == 'tmp':
        rng = tmp_ranges.get(id(o))
        if rng is None:
          raise GenerationError(f'temporary {o.name} is read before it is written')
        ref.origin = [l for l, _ in rng]
        ref.strides = _colmajor_strides([u - l for l, u in rng])
      elif o.kind in ('batched', 'shared'):
        ref.origin = list(o.bbox.lower())
        compact = identity and (0 not in ref.target)
        sizes = o.bbox.sizes() if compact else list(o.shape)
        ref.strides = _colmajor_strides(sizes)
      else:
        ref.origin = [0] * len(ref.target)
        ref.strides = [0] * len(ref.target)
    if dest.kind == 'tmp':
      tmp_ranges[id(dest)] = list(n_ranges)
      st.dest_origin = [l for l, _ in n_ranges]
      st.dest_strides = _colmajor_strides([u - l for l, u in n_ranges])
    else:
      st.dest_origin = list(dest.bbox.lower())
      st.dest_strides = _colmajor_strides(list(dest.shape))
    stages.append(st)
  return Chain(operands, tmps, stages, fp)
