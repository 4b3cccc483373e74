"""yateto layout -> Tensor conversion (tensorforge/interface.py:5-58)."""
from .common.matrix.tensor import Tensor
from .common.matrix.boundingbox import BoundingBox
from .common.matrix.spp import ListSPP


class YatetoInterface:
  @classmethod
  def deduce_bbox(cls, yateto_ranges, mem_layout, permute):
    """yateto memory-layout ranges -> bounding box (lower = range starts, upper = range stops)."""
    return BoundingBox([rng.start for rng in mem_layout], [rng.stop for rng in mem_layout])

  @classmethod
  def gen_matrix(cls, yateto_ranges, yateto_memory_layout_bbox, addressing, name, is_tmp, permute,
                 pattern=None, values=None, datatype=None):
    shape = [yateto_ranges[i] for i in range(len(yateto_ranges))]
    spp = ListSPP(pattern, tuple(shape)) if pattern is not None else None
    bbox = cls.deduce_bbox(yateto_ranges, yateto_memory_layout_bbox, permute)
    return Tensor(shape=shape, addressing=addressing, bbox=bbox, alias=name, is_tmp=is_tmp,
                  spp=spp, data=values, datatype=datatype)
