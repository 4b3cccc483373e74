"""Helpers for intermediate operands (tensorforge/common/aux.py:7-27)."""
from typing import List
from .matrix.tensor import Tensor, SubTensor
from .basic_types import Addressing, GeneralLexicon


def generate_tmp_tensor(ops: List[SubTensor], target: List[List[int]], alias=None):
  """Shape of the result of `ops` contracted by `target` (aux.py:7-22).

  Output dimension t takes the bounding-box extent of the operand dimension mapped to
  it; the result is a batched temporary that never appears in the launcher ABI.
  """
  rank = 0
  for itarget in target:
    for jtarget in itarget:
      rank = max(jtarget + 1, rank)
  shape = [0] * rank
  for i, itarget in enumerate(target):
    for j, jtarget in enumerate(itarget):
      if jtarget >= 0:
        shape[jtarget] = ops[i].bbox.sizes()[j]
  return Tensor(shape=shape, addressing=Addressing.PTR_BASED, bbox=None, is_tmp=True, alias=alias)


def generate_tmp_matrix(op1, op2, trans_a: bool = False, trans_b: bool = False):
  """Matrix-product temporary (aux.py:24-27); returns a SubTensor so it chains directly."""
  target_a = [-1, 0] if trans_a else [0, -1]
  target_b = [1, -1] if trans_b else [-1, 1]
  a = op1 if isinstance(op1, SubTensor) else SubTensor(op1)
  b = op2 if isinstance(op2, SubTensor) else SubTensor(op2)
  return SubTensor(generate_tmp_tensor([a, b], [target_a, target_b]))


def get_extra_offset_name(symbol):
  return f'{symbol.name}{GeneralLexicon.EXTRA_OFFSET}'
