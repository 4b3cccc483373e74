"""Elementwise statement trees (tensorforge/generators/optree.py:25-785).

An `ElementwiseDescr` holds a list of statements that run, for every batch element, at
every point (n0, n1, ...) of an index box:

    Assignment(dest, expr)        dest = expr
    IfNode(cond, statements)      if (cond) { statements }
    WhileNode(cond, statements)   while (cond) { statements }

Expressions are trees of `TensorVar` (a tensor read at the point), `ScalarVar` (a scalar
argument), `TempVar` (a per-point temporary), `Immediate` (a literal) and operation nodes
(`LexicOpNode` for the `Operation`s, `ConditionalOpNode` for `c ? a : b`, `CastOpNode`).
Python operators on nodes build trees (`a + b`, `a < b`, `-a`, `a ** 2`, ...), as do the
functions below (`exp`, `max`, `ternary`, `assign`, `conditional`, `loop`, ...), with the
reference's names and its algebraic shortcuts (`x * 1 -> x`, `x ** 0.5 -> sqrt(x)`, ...).

A `TensorVar` reads dimension j of its tensor at index n_{-indices[j]-1}: `indices` holds
negative numbers, -1 for n0, -2 for n1, like the contracted indices of a multilinear
target. The point (n0, ...) is relative to the tensor view's box: the entry read is
`bbox.lower + n`, and each n_i runs over [0, the smallest box size among the tensors it
indexes) (optree.py:229-238, elementwise.py:29-44).

Binding: a `TensorVar` made from a yateto node (`tensor(node)`) is bound later by the
frontend through `assignTensor(assigner)`, which returns the SubTensor and the index list
(frontend/yateto.py:127-148). A `TensorVar` can also be made bound directly from a
SubTensor or Tensor: `tensor(sub, indices=[-1, -2])` (default: -1, -2, ... over its rank).

Defined semantics where the reference leaves them open (its elementwise path does not
emit code): temporaries start at zero; float literals take the kernel's precision;
boolean operands make AND / OR / XOR / NOT the logical operators, integer ones the
bitwise ones; a `while` runs at most 2**24 iterations per point.
"""
import builtins
import math
from typing import List, Union

from ..common.basic_types import FloatingPointType
from ..common.exceptions import GenerationError
from ..common.operation import Operation
from ..common.matrix.tensor import Tensor, SubTensor

WHILE_LIMIT = 1 << 24


class Node:
  """Expression node. Python operators build operation nodes."""
  __hash__ = object.__hash__  # identity: `==` builds a comparison node

  def tensors(self, intensors=True, outtensors=True):
    return []

  def pretensors(self, intensors=True, outtensors=True):
    return []

  def getRanges(self, ranges):
    return ranges

  def assignTensor(self, assigner):
    pass

  def children(self):
    return []

  def __bool__(self):
    raise TypeError('an expression node has no truth value; use conditional() or ternary()')

  def __add__(self, other):
    return add(self, other)

  def __radd__(self, other):
    return add(other, self)

  def __sub__(self, other):
    return sub(self, other)

  def __rsub__(self, other):
    return sub(other, self)

  def __mul__(self, other):
    return mul(self, other)

  def __rmul__(self, other):
    return mul(other, self)

  def __truediv__(self, other):
    return div(self, other)

  def __rtruediv__(self, other):
    return div(other, self)

  def __mod__(self, other):
    return mod(self, other)

  def __rmod__(self, other):
    return mod(other, self)

  def __or__(self, other):
    return bitor(self, other)

  def __ror__(self, other):
    return bitor(other, self)

  def __and__(self, other):
    return bitand(self, other)

  def __rand__(self, other):
    return bitand(other, self)

  def __xor__(self, other):
    return bitxor(self, other)

  def __rxor__(self, other):
    return bitxor(other, self)

  def __invert__(self):
    return bitnot(self)

  def __pow__(self, other):
    return pow(self, other)

  def __rpow__(self, other):
    return pow(other, self)

  def __lt__(self, other):
    return complt(self, other)

  def __le__(self, other):
    return comple(self, other)

  def __gt__(self, other):
    return compgt(self, other)

  def __ge__(self, other):
    return compge(self, other)

  def __eq__(self, other):
    return compeq(self, other)

  def __ne__(self, other):
    return compne(self, other)

  def __neg__(self):
    return neg(self)

  def __pos__(self):
    return self

  def __abs__(self):
    return abs(self)


class Variable(Node):
  """A node that can also be assigned to."""


class Statement:
  __hash__ = object.__hash__

  def tensors(self, intensors=True, outtensors=True):
    return []

  def pretensors(self, intensors=True, outtensors=True):
    return []

  def getRanges(self, ranges):
    return ranges

  def assignTensor(self, assigner):
    pass

  def statements(self):
    return []


def _default_indices(sub):
  return [-(i + 1) for i in range(sub.bbox.rank())]


class TensorVar(Variable):
  def __init__(self, tensor, slicing=None, pretensor=None, indices=None):
    if isinstance(tensor, Tensor):
      tensor = SubTensor(tensor)
    self.tensor = tensor
    self.slicing = slicing
    self.pretensor = pretensor
    self.indices = None
    if tensor is not None:
      self.indices = list(indices) if indices is not None else _default_indices(tensor)

  def tensors(self, intensors=True, outtensors=True):
    if self.tensor is None:
      raise GenerationError('tensor variable is not bound to a tensor (assignTensor was not called)')
    return [self.tensor]

  def pretensors(self, intensors=True, outtensors=True):
    return [self.pretensor] if self.pretensor is not None else []

  def getRanges(self, ranges):
    """Index i -> (0, smallest box size among the dimensions it indexes) (optree.py:229-238)."""
    for j, idx in enumerate(self.indices):
      size = self.tensor.bbox.size(j)
      lo, up = ranges.get(idx, (0, size))
      ranges[idx] = (0, builtins.min(up, size))  # this module's min builds a node
    return ranges

  def assignTensor(self, assigner):
    if self.pretensor is not None:
      self.tensor, indices = assigner(self.pretensor)
      self.indices = list(indices)

  @property
  def offset(self):
    return list(self.tensor.bbox.lower())

  def __str__(self):
    idx = ','.join(f'n{-i - 1}' for i in (self.indices or []))
    return f'{self.tensor}[{idx}]'


class ScalarVar(Variable):
  """A rank-0 tensor: a by-value SCALAR argument or a compile-time value."""

  def __init__(self, tensor, slicing=None, pretensor=None):
    if isinstance(tensor, Tensor):
      tensor = SubTensor(tensor)
    self.tensor = tensor
    self.slicing = slicing
    self.pretensor = pretensor
    self.indices = [] if tensor is not None else None

  def tensors(self, intensors=True, outtensors=True):
    if self.tensor is None:
      raise GenerationError('scalar variable is not bound to a tensor (assignTensor was not called)')
    return [self.tensor]

  def assignTensor(self, assigner):
    if self.pretensor is not None:
      self.tensor, indices = assigner(self.pretensor)
      self.indices = list(indices)

  def __str__(self):
    return f'{self.tensor}'


class TempVar(Variable):
  """A per-point temporary (starts at zero)."""

  def __init__(self, datatype=None):
    self.datatype = datatype
    self.label = None

  def __str__(self):
    return self.label or 'temp'


class Immediate(Variable):
  def __init__(self, value, fptype: FloatingPointType):
    self.value = value
    self.fptype = fptype

  def __str__(self):
    return f'{self.value!r}'


class OpNode(Node):
  def __init__(self, operands: List[Node]):
    self.operands = list(operands)

  def children(self):
    return self.operands

  def getRanges(self, ranges):
    for op in self.operands:
      ranges = op.getRanges(ranges)
    return ranges

  def tensors(self, intensors=True, outtensors=True):
    return [t for op in self.operands for t in op.tensors()]

  def pretensors(self, intensors=True, outtensors=True):
    return [t for op in self.operands for t in op.pretensors()]

  def assignTensor(self, assigner):
    for op in self.operands:
      op.assignTensor(assigner)


class LexicOpNode(OpNode):
  def __init__(self, operands: List[Node], optype: Operation):
    super().__init__(operands)
    self.optype = optype

  def __str__(self):
    return f'{self.optype.name.lower()}({", ".join(str(o) for o in self.operands)})'


class ConditionalOpNode(OpNode):
  def __str__(self):
    c, a, b = self.operands
    return f'({c} ? {a} : {b})'


class CastOpNode(OpNode):
  def __init__(self, operands: List[Node], targetType: FloatingPointType):
    super().__init__(operands)
    self.targetType = targetType

  def __str__(self):
    return f'cast<{self.targetType}>({self.operands[0]})'


class Assignment(Statement):
  def __init__(self, dest: Variable, optree: Node):
    self.dest = dest
    self.optree = optree

  def tensors(self, intensors=True, outtensors=True):
    out = []
    if intensors:
      out += self.optree.tensors(intensors, outtensors)
    if outtensors:
      out += self.dest.tensors(intensors, outtensors)
    return out

  def pretensors(self, intensors=True, outtensors=True):
    out = []
    if intensors:
      out += self.optree.pretensors(intensors, outtensors)
    if outtensors:
      out += self.dest.pretensors(intensors, outtensors)
    return out

  def getRanges(self, ranges):
    ranges = self.dest.getRanges(ranges)
    return self.optree.getRanges(ranges)

  def assignTensor(self, assigner):
    self.dest.assignTensor(assigner)
    self.optree.assignTensor(assigner)

  def __str__(self):
    return f'{self.dest} = {self.optree}'


class _Block(Statement):
  def __init__(self, condition: Node, subassignments: List[Statement]):
    self.condition = condition
    self.subassignments = list(subassignments)

  def statements(self):
    return self.subassignments

  def getRanges(self, ranges):
    ranges = self.condition.getRanges(ranges)
    for s in self.subassignments:
      ranges = s.getRanges(ranges)
    return ranges

  def assignTensor(self, assigner):
    self.condition.assignTensor(assigner)
    for s in self.subassignments:
      s.assignTensor(assigner)

  def tensors(self, intensors=True, outtensors=True):
    out = self.condition.tensors(intensors, outtensors) if intensors else []
    return out + [t for s in self.subassignments for t in s.tensors(intensors, outtensors)]

  def pretensors(self, intensors=True, outtensors=True):
    out = self.condition.pretensors(intensors, outtensors) if intensors else []
    return out + [t for s in self.subassignments for t in s.pretensors(intensors, outtensors)]


class IfNode(_Block):
  def __str__(self):
    return f'if ({self.condition}) {{ {"; ".join(str(s) for s in self.subassignments)} }}'


class WhileNode(_Block):
  def __str__(self):
    return f'while ({self.condition}) {{ {"; ".join(str(s) for s in self.subassignments)} }}'


# ---------------------------------------------------------------------- tree walks
def walk_statements(statements):
  """Every statement, depth first, in program order."""
  for s in statements:
    yield s
    yield from walk_statements(s.statements())


def walk_nodes(node):
  yield node
  for c in node.children():
    yield from walk_nodes(c)


def statement_exprs(s):
  """Expression roots of one statement: the value and the target, or the condition."""
  if isinstance(s, Assignment):
    return [s.optree, s.dest]
  return [s.condition]


def label_temporaries(statements):
  """Name the temporaries v0, v1, ... in first-appearance order (stable kernel names)."""
  n = 0
  seen = set()
  for s in walk_statements(statements):
    for root in statement_exprs(s):
      for node in walk_nodes(root):
        if isinstance(node, TempVar) and id(node) not in seen:
          seen.add(id(node))
          node.label = f'v{n}'
          n += 1


# ---------------------------------------------------------------------- builders
BaseType = Union[Node, float, int, bool]


def _is_frontend_node(x):
  """A yateto tensor node (bound later through assignTensor)."""
  return hasattr(x, 'memoryLayout') or hasattr(x, 'eqspp')


def _is_frontend_scalar(x):
  return callable(getattr(x, 'name', None)) and not hasattr(x, 'memoryLayout')


def imm(value, fptype):
  return Immediate(value, fptype)


def immc(x: BaseType):
  if isinstance(x, bool):
    return imm(x, FloatingPointType.BOOL)
  if isinstance(x, int):
    return imm(x, FloatingPointType.INT)
  if isinstance(x, float):
    return imm(x, FloatingPointType.FLOAT)
  if isinstance(x, (Tensor, SubTensor)):
    sub = x if isinstance(x, SubTensor) else SubTensor(x)
    return scalar(sub) if sub.bbox.rank() == 0 else tensor(sub)
  if isinstance(x, Node):
    return x
  if _is_frontend_node(x):
    return tensor(x)
  if _is_frontend_scalar(x):
    return scalar(x)
  raise GenerationError(f'cannot use {x!r} in an elementwise expression')


def tensor(x, slicing=None, indices=None):
  if isinstance(x, (Tensor, SubTensor)):
    return TensorVar(x, slicing, None, indices)
  return TensorVar(None, slicing, x)


def scalar(x):
  if isinstance(x, (Tensor, SubTensor)):
    return ScalarVar(x)
  return ScalarVar(None, None, x)


def temp(datatype=None):
  return TempVar(datatype)


def assign(target, source: BaseType):
  if not isinstance(target, Variable):
    target = immc(target)
  return Assignment(target, immc(source))


def conditional(condition: BaseType, subnodes: List[Statement]):
  return IfNode(immc(condition), subnodes)


def loop(condition: BaseType, subnodes: List[Statement]):
  return WhileNode(immc(condition), subnodes)


def ternary(condition: BaseType, yesnode: BaseType, nonode: BaseType):
  return ConditionalOpNode([immc(condition), immc(yesnode), immc(nonode)])


def cast(x: BaseType, fptype: FloatingPointType):
  return CastOpNode([immc(x)], fptype)


def _unary(op):
  def f(x: BaseType):
    return LexicOpNode([immc(x)], op)
  f.__name__ = op.name.lower()
  return f


def _binary(op):
  def f(x: BaseType, y: BaseType):
    return LexicOpNode([immc(x), immc(y)], op)
  f.__name__ = op.name.lower()
  return f


cos, sin, tan = _unary(Operation.COS), _unary(Operation.SIN), _unary(Operation.TAN)
acos, asin, atan = _unary(Operation.ACOS), _unary(Operation.ASIN), _unary(Operation.ATAN)
cosh, sinh, tanh = _unary(Operation.COSH), _unary(Operation.SINH), _unary(Operation.TANH)
acosh, asinh, atanh = _unary(Operation.ACOSH), _unary(Operation.ASINH), _unary(Operation.ATANH)
sqrt, cbrt, rsqrt, rcbrt = _unary(Operation.SQRT), _unary(Operation.CBRT), _unary(Operation.RSQRT), _unary(Operation.RCBRT)
exp, log, expm1, logp1 = _unary(Operation.EXP), _unary(Operation.LOG), _unary(Operation.EXPM1), _unary(Operation.LOGP1)
round, rcp, abs = _unary(Operation.ROUND), _unary(Operation.RCP), _unary(Operation.ABS)
ceil, floor, trunc, sign = _unary(Operation.CEIL), _unary(Operation.FLOOR), _unary(Operation.TRUNC), _unary(Operation.SIGN)
erf, gamma = _unary(Operation.ERF), _unary(Operation.GAMMA)
neg, bitnot = _unary(Operation.NEG), _unary(Operation.NOT)
max, min, add, sub = _binary(Operation.MAX), _binary(Operation.MIN), _binary(Operation.ADD), _binary(Operation.SUB)
mod = _binary(Operation.MOD)
bitand, bitor, bitxor = _binary(Operation.AND), _binary(Operation.OR), _binary(Operation.XOR)
complt, comple = _binary(Operation.LT), _binary(Operation.LE)
compgt, compge = _binary(Operation.GT), _binary(Operation.GE)
compeq, compne = _binary(Operation.EQ), _binary(Operation.NEQ)


def _is_imm(x, *values):
  return isinstance(x, Immediate) and not isinstance(x.value, bool) and any(x.value == v for v in values)


def mul(x: BaseType, y: BaseType):
  """x * y, with 1 * y -> y and -1 * y -> -y (and mirrored) (optree.py:646-660)."""
  x, y = immc(x), immc(y)
  if _is_imm(x, 1):
    return y
  if _is_imm(x, -1):
    return neg(y)
  if _is_imm(y, 1):
    return x
  if _is_imm(y, -1):
    return neg(x)
  return LexicOpNode([x, y], Operation.MUL)


def div(x: BaseType, y: BaseType):
  """x / y, with 1 / y -> rcp(y), -1 / y -> rcp(-y), x / 1 -> x, x / -1 -> -x (optree.py:662-676)."""
  x, y = immc(x), immc(y)
  if _is_imm(x, 1):
    return LexicOpNode([y], Operation.RCP)
  if _is_imm(x, -1):
    return LexicOpNode([neg(y)], Operation.RCP)
  if _is_imm(y, 1):
    return x
  if _is_imm(y, -1):
    return neg(x)
  return LexicOpNode([x, y], Operation.DIV)


def pow(x: BaseType, y: BaseType):
  """x ** y with the reference's shortcuts (optree.py:692-715): y = 2 -> x*x, 0.5 -> sqrt,
  -0.5 -> rsqrt, 1/3 -> cbrt, -1/3 -> rcbrt, -1 -> rcp, 1 -> x; e ** y -> exp(y), 1 ** y -> 1."""
  x, y = immc(x), immc(y)
  if isinstance(y, Immediate) and not isinstance(y.value, bool):
    v = y.value
    if v == 2:
      return LexicOpNode([x, x], Operation.MUL)
    if v == 0.5:
      return LexicOpNode([x], Operation.SQRT)
    if v == -0.5:
      return LexicOpNode([x], Operation.RSQRT)
    if v == 1 / 3:
      return LexicOpNode([x], Operation.CBRT)
    if v == -1 / 3:
      return LexicOpNode([x], Operation.RCBRT)
    if v == -1:
      return LexicOpNode([x], Operation.RCP)
    if v == 1:
      return x
  if isinstance(x, Immediate) and not isinstance(x.value, bool):
    if x.value == math.e:
      return LexicOpNode([y], Operation.EXP)
    if x.value == 1:
      return x
  return LexicOpNode([x, y], Operation.POW)
