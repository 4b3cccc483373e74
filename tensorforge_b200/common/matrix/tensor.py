"""Operand descriptors (tensorforge/common/matrix/tensor.py:8-142).

A `Tensor` is one operand of a batched contraction: its shape, how each batch element's
copy is addressed, which sub-box holds data (`bbox`), which entries are nonzero (`spp`)
and, optionally, compile-time values (`data`). Memory layout is column-major over the
full shape with the origin at the bounding box's lower corner: entry `idx` of a dense
operand lives at `sum_j (idx_j - bbox.lower_j) * prod_{j'<j} shape_j'`. A sparse operand
stores only its nonzeros, compactly, at `spp.linear_index(idx - bbox.lower)`.
"""
from functools import reduce
from typing import List, Union
from .spp import SparsityPattern, FullSPP
from .boundingbox import BoundingBox
from ..basic_types import Addressing, DataFlowDirection, FloatingPointType
from ..exceptions import GenerationError


class Tensor:
  def __init__(self,
               shape: List[int],
               addressing: Addressing,
               bbox: Union[BoundingBox, None] = None,
               alias: Union[str, None] = None,
               is_tmp: bool = False,
               spp: SparsityPattern = None,
               data=None,
               datatype: FloatingPointType = None):
    self.name = None
    self.alias = alias
    self.shape = tuple(int(s) for s in shape)
    self.is_tmp = is_tmp
    self.direction: Union[DataFlowDirection, None] = None
    self.data = data
    self.spp = spp if spp is not None else FullSPP(self.shape)
    self.datatype = datatype
    self.bbox = bbox if bbox is not None else BoundingBox([0] * len(self.shape), self.shape)
    self.addressing = addressing
    self.ptr_type = self.addressing.to_pointer()

    if self.addressing == Addressing.SCALAR:
      assert all(d == 1 for d in self.shape)

    if any(s < b for s, b in zip(self.shape, self.bbox.sizes())):
      raise GenerationError(f'Tensor {self} is smaller than bounding box {self.bbox}')
    if any(s < u for s, u in zip(self.shape, self.bbox.upper())):
      raise GenerationError(f'Bounding box {self.bbox} is smaller than tensor {self}')

  def set_data_flow_direction(self, direction: DataFlowDirection):
    if self.direction is None or self.direction == direction:
      self.direction = direction
    else:
      self.direction = DataFlowDirection.SOURCESINK

  def has_values(self):
    return self.data is not None

  def get_values(self):
    return self.data

  def value(self, index):
    """Compile-time value at `index`, or None (tensor.py:57-62: `data` maps index tuples)."""
    key = tuple(index)
    if isinstance(self.data, dict) and key in self.data:
      return self.data[key]
    return None

  def linear_index(self, index):
    return self.spp.linear_index(tuple(index))

  def memory(self):
    return self.spp.count_nz()

  def get_actual_shape(self):
    return self.bbox.sizes()

  def get_actual_volume(self):
    return reduce(lambda x, y: x * y, self.get_actual_shape(), 1)

  def get_real_shape(self):
    return self.shape

  def get_real_volume(self):
    return reduce(lambda x, y: x * y, self.get_real_shape(), 1)

  def get_offset_to_first_element(self):
    return '0'

  def get_bbox(self):
    return self.bbox

  def _set_name(self, name):
    self.name = name

  def is_similar(self, other):
    return (self.shape == other.shape and self.addressing == other.addressing
            and self.bbox == other.bbox)

  def is_same(self, other):
    return self.is_similar(other)

  def is_dense(self):
    return self.spp.count_nz() == self.get_real_volume()

  def is_sparse_storage(self):
    """True if the operand is stored as a compact nonzero list (symbol.py:404)."""
    from .spp import BoundingBoxSPP
    return not self.is_dense() and not isinstance(self.spp, BoundingBoxSPP)

  def density(self):
    return self.spp.count_nz() / max(1, self.get_real_volume())

  def sparsity(self):
    return 1 - self.density()

  def gen_descr(self):
    return (f'{self.name} {"×".join(str(d) for d in self.shape)}'
            f'({"×".join(str(d) for d in self.bbox.sizes())}) {self.bbox} {self.addressing}')

  def __str__(self):
    return self.gen_descr()

  def __repr__(self):
    return self.gen_descr()


class TensorWrapper:
  pass


class SubTensor(TensorWrapper):
  """A view of a tensor restricted to `bbox` (tensor.py:129-142)."""

  def __init__(self, tensor: Tensor, bbox: Union[BoundingBox, None] = None):
    self.tensor = tensor
    self.bbox = bbox if bbox is not None else tensor.bbox

  def __str__(self):
    return f'{self.tensor}({self.bbox})'

  def __repr__(self):
    return str(self)


class FullTensor(TensorWrapper):
  def __init__(self, tensor: Tensor):
    self.tensor = tensor
