"""Operation descriptors (tensorforge/generators/descriptions.py:11-160).

`MultilinearDescr(dest, ops, target, permute, add)` describes, for every batch element,

    dest[n_0..n_{r-1}] (+)= sum_{k...} prod_i ops[i][idx_i]

where `target[i][j] >= 0` maps dimension j of operand i to output index n_t and
`target[i][j] < 0` maps it to the contracted index k_{-t-1}. Index ranges are the
intersections of the operands' bounding boxes. `permute[i][d]` is the stored dimension
of operand i that `target[i][d]` indexes (how `GemmDescr` expresses transposes).

`ElementwiseDescr(statements)` describes pointwise statements (see `optree`) over an
index box; both kinds can be mixed in one descriptor list.
"""
from typing import List
from ..common.exceptions import GenerationError
from ..common.basic_types import DataFlowDirection, Addressing, FloatingPointType  # noqa: F401 (re-exported)
from ..common.matrix.tensor import Tensor, SubTensor


class OperationDescription:
  pass


class MultilinearDescr(OperationDescription):
  def __init__(self, dest: SubTensor, ops: List[SubTensor], target, permute, add: bool = False,
               strict_match: bool = False, prefer_align: bool = False):
    self.dest = dest
    self.ops = ops
    self.target = [list(t) for t in target]
    self.permute = [list(p) for p in permute] if permute is not None else [list(range(len(t))) for t in target]
    self._strict_match = False
    self.add = add
    if len(self.target) != len(self.ops):
      raise GenerationError('target must have one entry per operand')
    for op, t in zip(self.ops, self.target):
      if len(t) != op.bbox.rank():
        raise GenerationError(f'target {t} does not match the rank of {op}')
    self.dest.tensor.set_data_flow_direction(DataFlowDirection.SINK)
    for op in self.ops:
      op.tensor.set_data_flow_direction(DataFlowDirection.SOURCE)

  def _lead_dim(self):
    sizes = self.dest.bbox.sizes()
    return sizes[0] if len(sizes) > 0 else 1

  def get_num_threads(self, context):
    lead = self._lead_dim()
    num_threads = context.align(num=lead)
    for cap in (32, 16, 8, 4, 2, 1):
      if lead <= cap:
        num_threads = cap
    return num_threads, lead

  def get_accumulator_size(self):
    acc = 1
    for s in self.dest.bbox.sizes()[1:]:
      acc *= s
    return acc

  def is_strict_match(self):
    return self._strict_match

  def matrix_list(self):
    return [self.dest] + list(self.ops)

  def __str__(self):
    desttarget = [i for i in range(self.dest.bbox.rank())]
    return f'{self.dest}{desttarget} = {"×".join(f"{op}{t}" for op, t in zip(self.ops, self.target))}'


class GemmDescr(MultilinearDescr):
  """C = alpha * A * B as a multilinear product (descriptions.py:126-149).

  The reference maps both transposes onto `permute` and keeps targets `[0,-1]`, `[-1,1]`;
  `beta` is accepted and ignored; alpha != 1 becomes an extra scalar operand carrying the
  value at generation time.
  """

  def __init__(self, trans_a, trans_b, a, b, c, alpha=1.0, beta=0.0,
               strict_match: bool = False, prefer_align: bool = False):
    target_a = [0, -1]
    target_b = [-1, 1]
    permute_a = [1, 0] if trans_a else [0, 1]
    permute_b = [1, 0] if trans_b else [0, 1]
    self.trans_a = trans_a
    self.trans_b = trans_b
    self.alpha = alpha
    self.beta = beta
    if alpha == 1.0:
      super().__init__(c, [a, b], [target_a, target_b], [permute_a, permute_b], strict_match, prefer_align)
    else:
      data = [alpha] if isinstance(alpha, (float, int)) else None
      alpha_tensor = SubTensor(Tensor([], Addressing.SCALAR, data=data))
      super().__init__(c, [a, b, alpha_tensor], [target_a, target_b, []],
                       [permute_a, permute_b, []], strict_match, prefer_align)


class ElementwiseDescr(OperationDescription):
  """Elementwise statements over an index box, per batch element (descriptions.py:67-95).

  `oplist` holds `optree` statements (`Assignment`, `IfNode`, `WhileNode`) whose tensor
  variables are bound. Tensors assigned to become SINK, tensors read become SOURCE (both:
  SOURCESINK), as in the reference. Stages of this kind can be mixed with
  `MultilinearDescr`s in one descriptor list: they read and write batched operands and
  temporaries, and a temporary written here can feed a later contraction.
  """

  def __init__(self, oplist, strict_match: bool = False, prefer_align: bool = False):
    from .optree import Statement, label_temporaries
    self.oplist = list(oplist)
    self._strict_match = False
    for op in self.oplist:
      if not isinstance(op, Statement):
        raise GenerationError(f'elementwise statements must be optree statements, got {type(op).__name__}')
    for op in self.oplist:
      for sub in op.tensors(outtensors=True, intensors=False):
        sub.tensor.set_data_flow_direction(DataFlowDirection.SINK)
    for op in self.oplist:
      for sub in op.tensors(outtensors=False, intensors=True):
        sub.tensor.set_data_flow_direction(DataFlowDirection.SOURCE)
    label_temporaries(self.oplist)

  def get_num_threads(self, context):
    return 64, 64

  def get_accumulator_size(self):
    return 0

  def is_strict_match(self):
    return self._strict_match

  def matrix_list(self):
    return [sub for op in self.oplist for sub in op.tensors()]

  def __str__(self):
    return '; '.join(str(op) for op in self.oplist)
