"""Sparsity patterns of an operand (tensorforge/common/matrix/spp.py:9-109).

A pattern says which entries can be nonzero and where the value of a nonzero is stored.
Sparse operands are stored compactly: only the nonzeros, in the pattern's own order
(`ListSPP`: the order of its entry list; `MaskSPP`: column-major order of the mask).
Indices passed to `linear_index` are relative to the tensor's bounding-box origin.
"""
from functools import reduce
import numpy as np


class SparsityPattern:
  @classmethod
  def from_values(cls, data, threshold=1):
    return None

  def nonzeros(self):
    """List of (relative index tuple, storage position), in storage order."""
    raise NotImplementedError


class FullSPP(SparsityPattern):
  def __init__(self, shape, permute=None):
    self.shape = tuple(shape)

  def is_nz(self, index):
    return True

  def count_nz(self):
    return reduce(lambda x, y: x * y, self.shape, 1)

  def linear_index(self, tupleindex):
    stride, index = 1, 0
    for x, s in zip(tupleindex, self.shape):
      index += x * stride
      stride *= s
    return index

  def dimrange(self, dim):
    return (0, self.shape[dim])

  def nonzeros(self):
    return [(tuple(int(v) for v in idx), self.linear_index(idx))
            for idx in _colmajor_indices(self.shape)]


class BoundingBoxSPP(SparsityPattern):
  def __init__(self, bbox):
    self.bbox = bbox

  def is_nz(self, index):
    return self.bbox.contains(index)

  def count_nz(self):
    return reduce(lambda x, y: x * y, self.bbox.sizes(), 1)

  def linear_index(self, tupleindex):
    stride, index = 1, 0
    for x, lo, up in zip(tupleindex, self.bbox.lower(), self.bbox.upper()):
      assert lo <= x < up
      index += (x - lo) * stride
      stride *= (up - lo)
    return index

  def dimrange(self, dim):
    return (self.bbox.lower()[dim], self.bbox.upper()[dim])

  def nonzeros(self):
    out = []
    for rel in _colmajor_indices(self.bbox.sizes()):
      idx = tuple(int(r + lo) for r, lo in zip(rel, self.bbox.lower()))
      out.append((idx, self.linear_index(idx)))
    return out


class MaskSPP(SparsityPattern):
  """Boolean mask pattern (spp.py:59-89).

  Storage positions follow the reference's construction: the mask is walked in its own
  memory order while positions are assigned in column-major order of the index mask.
  For a Fortran-ordered mask this is plain column-major numbering.
  """

  def __init__(self, mask):
    self.mask = np.asarray(mask)
    walk = self.mask.ravel(order='K').astype(bool)
    flat = np.zeros(walk.size, dtype=np.int64)
    flat[walk] = np.arange(1, int(walk.sum()) + 1)
    self.indexmask = flat.reshape(self.mask.shape, order='F')

  def is_nz(self, index):
    return bool(self.mask[tuple(index)])

  def count_nz(self):
    return int(np.count_nonzero(self.mask))

  def linear_index(self, tupleindex):
    if all(ti < ims for ti, ims in zip(tupleindex, self.indexmask.shape)):
      pre = int(self.indexmask[tuple(tupleindex)])
      return pre - 1 if pre > 0 else None
    return None

  def dimrange(self, dim):
    return None

  def nonzeros(self):
    pos = np.argwhere(self.indexmask > 0)
    items = [(tuple(int(v) for v in p), int(self.indexmask[tuple(p)]) - 1) for p in pos]
    return sorted(items, key=lambda kv: kv[1])


class ListSPP(SparsityPattern):
  """Explicit entry list; the value of entry n is stored at compact position n."""

  def __init__(self, lst, shape):
    self.list = [tuple(int(v) for v in e) for e in lst]
    self.shape = tuple(shape)
    self.indexmask = np.zeros(self.shape, dtype=np.int64, order='F')
    for i, entry in enumerate(self.list):
      self.indexmask[entry] = i + 1

  def is_nz(self, index):
    return self.indexmask[tuple(index)] > 0

  def count_nz(self):
    return int(np.count_nonzero(self.indexmask))

  def linear_index(self, tupleindex):
    if all(ti < ims for ti, ims in zip(tupleindex, self.indexmask.shape)):
      pre = int(self.indexmask[tuple(tupleindex)])
      return pre - 1 if pre > 0 else None
    return None

  def dimrange(self, dim):
    return None

  def nonzeros(self):
    # a repeated entry keeps its last position, like the index mask built above
    seen = {}
    for i, e in enumerate(self.list):
      seen[e] = i
    return sorted(seen.items(), key=lambda kv: kv[1])


def _colmajor_indices(shape):
  shape = list(shape)
  if len(shape) == 0:
    return [()]
  total = reduce(lambda x, y: x * y, shape, 1)
  idx = np.unravel_index(np.arange(total), shape, order='F')
  return list(zip(*[i.tolist() for i in idx]))
