"""Half-open index boxes `[lower, upper)` per dimension (tensorforge/common/matrix/boundingbox.py:3-50)."""
from typing import List


class BoundingBox:
  def __init__(self, lower: List[int], upper: List[int]):
    assert len(lower) == len(upper)
    self._lower = tuple(int(x) for x in lower)
    self._upper = tuple(int(x) for x in upper)

  def intersect(self, other):
    return BoundingBox([max(a, b) for a, b in zip(self._lower, other._lower)],
                       [min(a, b) for a, b in zip(self._upper, other._upper)])

  def unite(self, other):
    return BoundingBox([min(a, b) for a, b in zip(self._lower, other._lower)],
                       [max(a, b) for a, b in zip(self._upper, other._upper)])

  def __rand__(self, other):
    return self.intersect(other)

  def __ror__(self, other):
    return self.unite(other)

  def __iter__(self):
    for lo, up in zip(self._lower, self._upper):
      yield lo, up

  def __eq__(self, other):
    return isinstance(other, BoundingBox) and self._lower == other._lower and self._upper == other._upper

  def __hash__(self):
    return hash((self._lower, self._upper))

  def rank(self):
    return len(self._lower)

  def contains(self, index):
    return all(lo <= i < up for i, lo, up in zip(index, self._lower, self._upper))

  def empty(self):
    return any(up <= lo for lo, up in zip(self._lower, self._upper))

  def lower(self):
    return self._lower

  def upper(self):
    return self._upper

  def size(self, dim):
    return self._upper[dim] - self._lower[dim]

  def sizes(self):
    return [up - lo for lo, up in zip(self._lower, self._upper)]

  def __str__(self):
    return '×'.join(f'{{{lo}..{up}}}' for lo, up in zip(self._lower, self._upper))

  def __repr__(self):
    return str(self)
