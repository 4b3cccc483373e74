"""CUDA emission of elementwise stages (used by the generic generator).

The lanes of an element's group split the points of the stage's index box
(d = lane, lane + G, ...); each point runs the statements in order, with its own
temporaries (zero-initialised). Every expression node becomes one `const` local
(the reference's optree writes the same single-assignment form, optree.py:402-409), typed
by a small inference: comparisons and logical operators give `bool`, integer literals
and integer-only arithmetic give `int`, everything else is the kernel's floating-point
type. Math functions are the CUDA math library's (`expf`/`exp`, ...); operation
spellings follow the reference's CUDA lexic (common/vm/lexic/cuda_lexic.py:113-206),
completed for the operations it leaves unimplemented (ceil, floor, round, trunc, sign,
rsqrt, rcbrt, mod, log1p).
"""
from ..common.basic_types import FloatingPointType as FP
from ..common.exceptions import GenerationError
from ..common.operation import Operation, UNARY_MATH, BINARY_MATH, ARITHMETIC, COMPARISON, BITWISE, LOGICAL
from ..generators import optree as ot

WHILE_LIMIT = ot.WHILE_LIMIT


def _colmajor(sizes):
  out, acc = [], 1
  for s in sizes:
    out.append(acc)
    acc *= s
  return out


class PointEmitter:
  """Emits the body of one point of an elementwise stage into a GenericEmitter."""

  def __init__(self, em, stage, sfx='', counter=None):
    self.em = em
    self.stage = stage
    self.fp = em.ctx.fp_type
    self.T = em.T
    self.sfx = sfx                      # name suffix of this point's indices and temporaries
    self.counter = counter if counter is not None else [0]
    self.memo = {}

  # ------------------------------------------------------------------ types
  def ctype(self, ty):
    return {'fp': self.T, 'int': 'int', 'bool': 'bool'}.get(ty, ty)

  def _fp(self, expr, ty):
    return expr if ty == 'fp' else f'static_cast<{self.T}>({expr})'

  def _mathname(self, base):
    return base + ('f' if self.fp == FP.FLOAT else '')

  # ------------------------------------------------------------------ operands
  def _index_exprs(self, acc):
    return [f'(n{d}{self.sfx} + {b})' for d, b in zip(acc.dims, acc.base)]

  def _address(self, acc):
    terms = [f'({e} - {org}) * {st}' for e, org, st in zip(self._index_exprs(acc), acc.origin, acc.strides)]
    return ' + '.join(terms) or '0'

  def lvalue(self, node):
    acc = self.stage.access[id(node)]
    o = acc.op
    if o.kind == 'tmp':
      return f'tmp_{o.name}[{self._address(acc)}]'
    return f'glb_{o.name}[{self._address(acc)}]'

  def load(self, node):
    acc = self.stage.access[id(node)]
    o = acc.op
    if o.kind == 'scalar':
      return o.name
    if o.kind == 'data':
      data = o.tensor.data
      if len(acc.dims) == 0:
        v = data.get((), 0.0) if isinstance(data, dict) else float(data[0])
        return self.em.lit(v)
      idx = self._index_exprs(acc)
      return f'data_{o.name}[{" + ".join(f"({e}) * {st}" for e, st in zip(idx, _colmajor(list(o.shape))))}]'
    if o.kind != 'tmp' and o.sparse:
      return f'dn_{o.name}[{self._address(acc)}]'
    return self.lvalue(node)

  # ------------------------------------------------------------------ expressions
  def expr(self, node):
    """(C expression naming the node's value, type) with one const local per operation."""
    key = id(node)
    if key in self.memo:
      return self.memo[key]
    out = self._expr(node)
    self.memo[key] = out
    return out

  def _local(self, ty, text):
    name = f'e{self.counter[0]}'
    self.counter[0] += 1
    self.em.w(f'const {self.ctype(ty)} {name} = {text};')
    return name

  def _expr(self, node):
    if isinstance(node, ot.Immediate):
      if node.fptype == FP.BOOL or isinstance(node.value, bool):
        return ('true' if node.value else 'false'), 'bool'
      if node.fptype in (FP.INT, FP.UINT, FP.LONG, FP.ULONG):
        return f'{int(node.value)}', 'int'
      return self.em.lit(node.value), 'fp'
    if isinstance(node, ot.TempVar):
      return node.label + self.sfx, self._temp_type(node)
    if isinstance(node, (ot.TensorVar, ot.ScalarVar)):
      return self._local('fp', self.load(node)), 'fp'
    if isinstance(node, ot.ConditionalOpNode):
      (c, ct), (a, at), (b, bt) = [self.expr(x) for x in node.operands]
      ty = 'fp' if 'fp' in (at, bt) else ('int' if 'int' in (at, bt) else 'bool')
      if ty == 'fp':
        a, b = self._fp(a, at), self._fp(b, bt)
      return self._local(ty, f'({c}) ? ({a}) : ({b})'), ty
    if isinstance(node, ot.CastOpNode):
      a, at = self.expr(node.operands[0])
      tgt = node.targetType
      ty = 'bool' if tgt == FP.BOOL else ('int' if tgt in (FP.INT, FP.UINT, FP.LONG, FP.ULONG) else str(tgt))
      if tgt == self.fp:
        ty = 'fp'
      return self._local(ty, f'static_cast<{self.ctype(ty)}>({a})'), ty
    if isinstance(node, ot.LexicOpNode):
      return self._op(node)
    raise GenerationError(f'unsupported expression node {type(node).__name__}')

  def _op(self, node):
    op = node.optype
    args = [self.expr(x) for x in node.operands]
    if op == Operation.COPY:
      return args[0]
    if op in ARITHMETIC:
      (a, at), (b, bt) = args
      if at != 'fp' and bt != 'fp':
        return self._local('int', f'{a} {ARITHMETIC[op]} {b}'), 'int'
      return self._local('fp', f'{self._fp(a, at)} {ARITHMETIC[op]} {self._fp(b, bt)}'), 'fp'
    if op == Operation.NEG:
      a, at = args[0]
      ty = 'fp' if at == 'fp' else 'int'
      return self._local(ty, f'-{a}'), ty
    if op == Operation.RCP:
      a, at = args[0]
      return self._local('fp', f'{self.em.lit(1.0)} / {self._fp(a, at)}'), 'fp'
    if op in UNARY_MATH:
      a, at = args[0]
      return self._local('fp', f'{self._mathname(UNARY_MATH[op])}({self._fp(a, at)})'), 'fp'
    if op == Operation.SIGN:
      a, at = args[0]
      x = self._fp(a, at)
      return self._local('fp', f'static_cast<{self.T}>(({x} > 0) - ({x} < 0))'), 'fp'
    if op == Operation.MOD and all(t != 'fp' for _, t in args):
      (a, _), (b, _) = args
      return self._local('int', f'{a} % {b}'), 'int'
    if op in BINARY_MATH:
      (a, at), (b, bt) = args
      return self._local('fp', f'{self._mathname(BINARY_MATH[op])}({self._fp(a, at)}, {self._fp(b, bt)})'), 'fp'
    if op in COMPARISON:
      (a, at), (b, bt) = args
      if 'fp' in (at, bt):
        a, b = self._fp(a, at), self._fp(b, bt)
      return self._local('bool', f'{a} {COMPARISON[op]} {b}'), 'bool'
    if op == Operation.NOT:
      a, at = args[0]
      if at == 'bool':
        return self._local('bool', f'!{a}'), 'bool'
      if at == 'int':
        return self._local('int', f'~{a}'), 'int'
      raise GenerationError('bitwise NOT of a floating-point value')
    if op in BITWISE or op in LOGICAL:
      (a, at), (b, bt) = args
      if at == 'bool' and bt == 'bool' and op in LOGICAL:
        return self._local('bool', f'{a} {LOGICAL[op]} {b}'), 'bool'
      if 'fp' in (at, bt):
        raise GenerationError(f'{op.name} of a floating-point value')
      return self._local('int', f'{a} {BITWISE[op]} {b}'), 'int'
    raise GenerationError(f'unsupported operation {op.name}')

  # ------------------------------------------------------------------ statements
  def _temp_type(self, node):
    dt = node.datatype
    if dt is None or dt == self.fp:
      return 'fp'
    if dt == FP.BOOL:
      return 'bool'
    if dt in (FP.INT, FP.UINT, FP.LONG, FP.ULONG):
      return 'int'
    return str(dt)

  def declare_temporaries(self):
    for t in self.stage.temporaries():
      ty = self._temp_type(t)
      zero = {'fp': self.em.lit(0.0), 'int': '0', 'bool': 'false'}.get(ty, '0')
      self.em.w(f'{self.ctype(ty)} {t.label}{self.sfx} = {zero};')

  def store(self, s, v, vt):
    if isinstance(s.dest, ot.TempVar):
      ty = self._temp_type(s.dest)
      val = self._fp(v, vt) if ty == 'fp' else f'static_cast<{self.ctype(ty)}>({v})'
      self.em.w(f'{s.dest.label}{self.sfx} = {val};')
    else:
      self.em.w(f'{self.lvalue(s.dest)} = {self._fp(v, vt)};')

  def statements(self, stmts, depth=0):
    for s in stmts:
      self.memo = {}  # values are re-read after every statement (it may have stored to them)
      if isinstance(s, ot.Assignment):
        self.store(s, *self.expr(s.optree))
      elif isinstance(s, ot.IfNode):
        with self.em.block(''):
          c, _ = self.expr(s.condition)
          with self.em.block(f'if ({c})'):
            self.statements(s.subassignments, depth + 1)
      elif isinstance(s, ot.WhileNode):
        g = f'w{depth}{self.sfx}'
        with self.em.block(f'for (unsigned {g} = 0; {g} < {WHILE_LIMIT}u; ++{g})'):
          c, _ = self.expr(s.condition)
          self.em.w(f'if (!({c})) break;')
          self.statements(s.subassignments, depth + 1)
      else:
        raise GenerationError(f'unsupported statement {type(s).__name__}')
      self.memo = {}


class RegisterPointEmitter(PointEmitter):
  """Point (row, column) of an elementwise epilogue whose output entry is a register.

  The chain's output `out` is read and written as `reg[row]`; other batched operands are
  read at the same entry of the element through `elem_ptr(op)` (column-major M x N);
  n0 = row (a constant), n1 = `col` (the thread's column)."""

  def __init__(self, em, stage, out, reg, row, col, M, elem_ptr, counter):
    super().__init__(em, stage, f'_{row}', counter)
    self.out, self.reg, self.row, self.col, self.M, self.elem_ptr = out, reg, row, col, M, elem_ptr

  def _index_exprs(self, acc):
    return [f'({self.row if d == 0 else self.col} + {b})' for d, b in zip(acc.dims, acc.base)]

  def lvalue(self, node):
    acc = self.stage.access[id(node)]
    if acc.op is not self.out:
      raise GenerationError(f'an epilogue writes the chain output only, not {acc.op.name}')
    return f'{self.reg}[{self.row}]'

  def load(self, node):
    acc = self.stage.access[id(node)]
    o = acc.op
    if o is self.out:
      return f'{self.reg}[{self.row}]'
    if o.kind == 'batched':
      return f'__ldg({self.elem_ptr(o)} + {self.row} + {self.col} * {self.M})'
    return super().load(node)


def multi_point_statements(em, pes, stmts):
  """Statements for several points at once, statement by statement: all points' values
  (their loads in flight together) before any point's store. Points never touch each
  other's entries (checked at lowering), so this order computes what running the points
  one after another computes. `if` and `while` bodies run point by point."""
  for s in stmts:
    for pe in pes:
      pe.memo = {}
    if isinstance(s, ot.Assignment):
      vals = [pe.expr(s.optree) for pe in pes]
      for pe, (v, vt) in zip(pes, vals):
        pe.store(s, v, vt)
    elif isinstance(s, ot.IfNode):
      conds = [pe.expr(s.condition)[0] for pe in pes]
      for pe, c in zip(pes, conds):
        with em.block(f'if ({c})'):
          pe.statements(s.subassignments, 1)
    else:
      for pe in pes:
        pe.statements([s])
    for pe in pes:
      pe.memo = {}


def emit_elementwise_stage(em, stage):
  """Point loop of one elementwise stage (inside the element's `if (active)`).

  The lanes of the group take points d = lane, lane + G, ...; a pass handles
  `points_per_lane` (U) points per lane at once, then single points finish the rest."""
  G = em.G
  U = int(em.plan.params.get('points_per_lane', 4))
  sizes = stage.sizes
  vol = 1
  for s in sizes:
    vol *= s
  counter = [0]

  def indices(d, sfx):
    div = 1
    for i, s in enumerate(sizes):
      expr = f'({d} / {div}u) % {s}u' if div > 1 else f'{d} % {s}u'
      em.w(f'const int n{i}{sfx} = (int)({expr});')
      div *= s

  em.w('unsigned d0 = lane;')
  if U > 1 and vol > G:
    with em.block(f'for (; d0 + {(U - 1) * G}u < {vol}u; d0 += {U * G}u)'):
      pes = []
      for u in range(U):
        indices(f'(d0 + {u * G}u)', f'_{u}')
        pe = PointEmitter(em, stage, f'_{u}', counter)
        pe.declare_temporaries()
        pes.append(pe)
      multi_point_statements(em, pes, stage.statements)
  with em.block(f'for (; d0 < {vol}u; d0 += {G}u)'):
    indices('d0', '')
    pe = PointEmitter(em, stage, '', counter)
    pe.declare_temporaries()
    pe.statements(stage.statements)
