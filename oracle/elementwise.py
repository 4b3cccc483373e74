"""FP64 restatement of elementwise statements (`ElementwiseDescr`), per batch element.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Follows the statement semantics of the reference's optree and ElementwiseInstruction:
  * the index box: n_i over [0, the smallest view-box size among the tensor dimensions it
    indexes): tensorforge/generators/optree.py:229-238,
    tensorforge/backend/instructions/compute/elementwise.py:29-44
  * a tensor variable reads / writes entry `view.bbox.lower + n` (optree.py:247-257) at the
    address sum_j (entry_j - tensor.bbox.lower_j) * stride_j over the tensor's shape, a
    sparse one its compact value (zero when absent), like multilinear operands:
    tensorforge/backend/symbol.py:304-330, :340-401
  * statements run in order at every point; `if` and `while` guard their statements
    (optree.py:402-409, :434-520); operations as spelled by the CUDA lexic
    (common/vm/lexic/cuda_lexic.py:113-206)
The reference's CUDA and OpenMP lexics cannot emit this path (its ElementwiseInstruction
stops with a TypeError), so these semantics are pinned by this restatement and the
hand-computed cases in the tests, not by reference outputs.

Evaluation is vectorised over (elements, points): points of one stage never touch each
other's entries (the generator rejects statements where they would), so running all
points at once is the same as running them one by one. Booleans stay numpy bool,
integers int64, floating-point values float64.
"""
import math

import numpy as np

from tensorforge_b200.common.basic_types import FloatingPointType as FP
from tensorforge_b200.common.operation import Operation
from tensorforge_b200.generators import optree as ot

WHILE_LIMIT = ot.WHILE_LIMIT


def _colmajor(sizes):
  out, acc = [], 1
  for s in sizes:
    out.append(acc)
    acc *= s
  return out


def _c_round(x):
  """C `round`: halves away from zero (numpy's round is half-to-even)."""
  return np.sign(x) * np.floor(np.abs(x) + 0.5)


_vgamma = np.vectorize(lambda v: math.gamma(v) if v > 0 or v != math.floor(v) else math.nan, otypes=[np.float64])
_verf = np.vectorize(math.erf, otypes=[np.float64])

UNARY = {
  Operation.SQRT: np.sqrt, Operation.CBRT: np.cbrt, Operation.RSQRT: lambda x: 1.0 / np.sqrt(x),
  Operation.RCBRT: lambda x: 1.0 / np.cbrt(x), Operation.ABS: np.abs, Operation.CEIL: np.ceil,
  Operation.FLOOR: np.floor, Operation.ROUND: _c_round, Operation.TRUNC: np.trunc, Operation.LOGP1: np.log1p,
  Operation.EXPM1: np.expm1, Operation.GAMMA: _vgamma, Operation.ERF: _verf, Operation.LOG: np.log,
  Operation.EXP: np.exp, Operation.SIN: np.sin, Operation.COS: np.cos, Operation.TAN: np.tan,
  Operation.ASIN: np.arcsin, Operation.ACOS: np.arccos, Operation.ATAN: np.arctan, Operation.SINH: np.sinh,
  Operation.COSH: np.cosh, Operation.TANH: np.tanh, Operation.ASINH: np.arcsinh, Operation.ACOSH: np.arccosh,
  Operation.ATANH: np.arctanh,
}


def _kind(v):
  dt = np.asarray(v).dtype
  if dt == np.bool_:
    return 'bool'
  if np.issubdtype(dt, np.integer):
    return 'int'
  return 'fp'


def _as_fp(v):
  return np.asarray(v, dtype=np.float64)


def _as_int(v):
  return np.asarray(v).astype(np.int64)


def _c_div_int(a, b):
  """C integer division (truncates toward zero)."""
  q = np.abs(a) // np.abs(b)
  return np.where((a < 0) != (b < 0), -q, q)


def _c_mod_int(a, b):
  return a - _c_div_int(a, b) * b


class _Stage:
  def __init__(self, descr, memory, elems, sym_names, tmp_values):
    self.memory = memory
    self.elems = elems
    self.ne = len(elems)
    self.sym = sym_names
    self.tmp_values = tmp_values
    ranges = {}
    for s in descr.oplist:
      ranges = s.getRanges(ranges)
    self.sizes = [ranges[-(i + 1)][1] for i in range(len(ranges))]
    self.shape = (self.ne,) + tuple(self.sizes)
    self.grid = np.meshgrid(*[np.arange(s) for s in self.sizes], indexing='ij') if self.sizes else []
    self.temps = {}

  # ---------------------------------------------------------------- entries
  def _entry(self, var):
    """Absolute index arrays (one per tensor dimension, broadcast over the points)."""
    base = var.tensor.bbox.lower()
    return [self.grid[-i - 1] + b for i, b in zip(var.indices, base)]

  def _dense_address(self, t, entry):
    name = self.sym[id(t)]
    addr_kind = str(t.addressing)
    start = np.zeros(self.ne, dtype=np.int64) if addr_kind == 'none' else np.asarray(self.memory.starts[name])[self.elems]
    off = np.zeros(self.sizes, dtype=np.int64)
    for e, lo, st in zip(entry, t.bbox.lower(), _colmajor(list(t.shape))):
      off = off + (e - lo) * st
    return start.reshape((-1,) + (1,) * len(self.sizes)) + off[None]

  def read(self, var):
    t = var.tensor.tensor
    if t.is_tmp:
      rng, arr = self.tmp_values[id(t)]
      entry = self._entry(var)
      rel = tuple(e - r0 for e, (r0, _) in zip(entry, rng))
      idx = (np.arange(self.ne).reshape((-1,) + (1,) * len(self.sizes)),) + tuple(r[None] for r in rel)
      return arr[idx] if rel else np.broadcast_to(arr.reshape((-1,) + (1,) * len(self.sizes)), self.shape)
    if str(t.addressing) == 'scalar':
      if t.data is not None and len(t.data) < 16:
        d = t.data
        v = float(d.get((), 0.0)) if isinstance(d, dict) else float(d[0])
      else:
        v = float(self.memory.scalars[self.sym[id(t)]])
      return np.full(self.shape, v)
    if t.data is not None and len(t.data) < 16:
      entry = self._entry(var)
      out = np.zeros(self.sizes)
      for p in np.ndindex(*self.sizes):
        v = t.value(tuple(int(e[p]) for e in entry))
        out[p] = 0.0 if v is None else v
      return np.broadcast_to(out[None], self.shape)
    name = self.sym[id(t)]
    buf = self.memory.buffers[name]
    entry = self._entry(var)
    spp = t.spp
    mask = getattr(spp, 'indexmask', None)
    dense = mask is None or int(np.count_nonzero(mask)) == int(np.prod(t.shape))
    if not dense:
      start = np.zeros(self.ne, dtype=np.int64) if str(t.addressing) == 'none' else np.asarray(self.memory.starts[name])[self.elems]
      rel = [e - lo for e, lo in zip(entry, t.bbox.lower())]
      pos = np.asarray(mask)[tuple(rel)].astype(np.int64) - 1
      vals = buf[start.reshape((-1,) + (1,) * len(self.sizes)) + np.maximum(pos, 0)[None]]
      return np.where(pos[None] >= 0, vals, 0.0)
    return buf[self._dense_address(t, entry)]

  def write(self, var, value, mask):
    t = var.tensor.tensor
    value = np.broadcast_to(_as_fp(value), self.shape)
    mask = np.broadcast_to(mask, self.shape)
    entry = self._entry(var)
    if t.is_tmp:
      if id(t) not in self.tmp_values:
        rng = [(int(b), int(b) + self.sizes[-i - 1]) for i, b in zip(var.indices, var.tensor.bbox.lower())]
        self.tmp_values[id(t)] = (rng, np.zeros((self.ne,) + tuple(u - l for l, u in rng)))
      rng, arr = self.tmp_values[id(t)]
      rel = tuple(np.broadcast_to(e - r0, self.sizes)[None] for e, (r0, _) in zip(entry, rng))
      el = np.broadcast_to(np.arange(self.ne).reshape((-1,) + (1,) * len(self.sizes)), self.shape)
      idx = (el,) + tuple(np.broadcast_to(r, self.shape) for r in rel)
      sel = tuple(i[mask] for i in idx)
      arr[sel] = value[mask]
      return
    buf = self.memory.buffers[self.sym[id(t)]]
    addr = np.broadcast_to(self._dense_address(t, entry), self.shape)
    buf[addr[mask]] = value[mask]

  # ---------------------------------------------------------------- expressions
  def eval(self, node, fp32):
    if isinstance(node, ot.Immediate):
      if node.fptype == FP.BOOL or isinstance(node.value, bool):
        return np.bool_(bool(node.value))
      if node.fptype in (FP.INT, FP.UINT, FP.LONG, FP.ULONG):
        return np.int64(int(node.value))
      return np.float64(node.value)
    if isinstance(node, ot.TempVar):
      return self.temps[id(node)]
    if isinstance(node, (ot.TensorVar, ot.ScalarVar)):
      return self.read(node)
    if isinstance(node, ot.ConditionalOpNode):
      c, a, b = [self.eval(x, fp32) for x in node.operands]
      if 'fp' in (_kind(a), _kind(b)):
        a, b = _as_fp(a), _as_fp(b)
      return np.where(c, a, b)
    if isinstance(node, ot.CastOpNode):
      a = self.eval(node.operands[0], fp32)
      tgt = node.targetType
      if tgt == FP.BOOL:
        return np.asarray(a) != 0
      if tgt in (FP.INT, FP.UINT, FP.LONG, FP.ULONG):
        return np.trunc(_as_fp(a)).astype(np.int64)
      if tgt == FP.FLOAT:
        return _as_fp(a).astype(np.float32).astype(np.float64)
      return _as_fp(a)
    return self._op(node, [self.eval(x, fp32) for x in node.operands])

  def _op(self, node, args):
    op = node.optype
    kinds = [_kind(a) for a in args]
    if op == Operation.COPY:
      return args[0]
    if op in (Operation.ADD, Operation.SUB, Operation.MUL, Operation.DIV):
      a, b = args
      if 'fp' not in kinds:
        a, b = _as_int(a), _as_int(b)
        return {Operation.ADD: a + b, Operation.SUB: a - b, Operation.MUL: a * b}[op] if op != Operation.DIV \
          else _c_div_int(a, b)
      a, b = _as_fp(a), _as_fp(b)
      return {Operation.ADD: np.add, Operation.SUB: np.subtract, Operation.MUL: np.multiply,
              Operation.DIV: np.divide}[op](a, b)
    if op == Operation.NEG:
      a = args[0]
      return -_as_fp(a) if kinds[0] == 'fp' else -_as_int(a)
    if op == Operation.RCP:
      return 1.0 / _as_fp(args[0])
    if op in UNARY:
      return UNARY[op](_as_fp(args[0]))
    if op == Operation.SIGN:
      x = _as_fp(args[0])
      return (x > 0).astype(np.float64) - (x < 0).astype(np.float64)
    if op == Operation.MOD:
      if 'fp' not in kinds:
        return _c_mod_int(_as_int(args[0]), _as_int(args[1]))
      return np.fmod(_as_fp(args[0]), _as_fp(args[1]))
    if op == Operation.MIN:
      return np.fmin(_as_fp(args[0]), _as_fp(args[1]))
    if op == Operation.MAX:
      return np.fmax(_as_fp(args[0]), _as_fp(args[1]))
    if op == Operation.POW:
      return np.power(_as_fp(args[0]), _as_fp(args[1]))
    if op in (Operation.EQ, Operation.NEQ, Operation.LT, Operation.LE, Operation.GT, Operation.GE):
      a, b = args
      if 'fp' in kinds:
        a, b = _as_fp(a), _as_fp(b)
      return {Operation.EQ: np.equal, Operation.NEQ: np.not_equal, Operation.LT: np.less,
              Operation.LE: np.less_equal, Operation.GT: np.greater, Operation.GE: np.greater_equal}[op](a, b)
    if op == Operation.NOT:
      a = args[0]
      return np.logical_not(a) if kinds[0] == 'bool' else ~_as_int(a)
    if op in (Operation.AND, Operation.OR, Operation.XOR):
      a, b = args
      if kinds == ['bool', 'bool']:
        return {Operation.AND: np.logical_and, Operation.OR: np.logical_or,
                Operation.XOR: np.logical_xor}[op](a, b)
      a, b = _as_int(a), _as_int(b)
      return {Operation.AND: a & b, Operation.OR: a | b, Operation.XOR: a ^ b}[op]
    if op in (Operation.SHL, Operation.SHR, Operation.SHRS):
      a, b = _as_int(args[0]), _as_int(args[1])
      return a << b if op == Operation.SHL else a >> b
    raise NotImplementedError(op)

  # ---------------------------------------------------------------- statements
  def run(self, statements, mask, fp32):
    for s in statements:
      if isinstance(s, ot.Assignment):
        v = self.eval(s.optree, fp32)
        if isinstance(s.dest, ot.TempVar):
          prev = self.temps[id(s.dest)]
          dt = prev.dtype
          if dt == np.bool_:
            v = np.asarray(v) != 0
          elif np.issubdtype(dt, np.integer):
            v = np.trunc(_as_fp(v)).astype(np.int64) if _kind(v) == 'fp' else _as_int(v)
          else:
            v = _as_fp(v)
            if fp32 or s.dest.datatype == FP.FLOAT:
              v = v.astype(np.float32).astype(np.float64)
          self.temps[id(s.dest)] = np.where(np.broadcast_to(mask, self.shape), np.broadcast_to(v, self.shape), prev)
        else:
          self.write(s.dest, v, mask)
      elif isinstance(s, ot.IfNode):
        c = np.broadcast_to(np.asarray(self.eval(s.condition, fp32)) != 0, self.shape)
        self.run(s.subassignments, mask & c, fp32)
      elif isinstance(s, ot.WhileNode):
        live = mask.copy()
        for _ in range(WHILE_LIMIT):
          live = live & np.broadcast_to(np.asarray(self.eval(s.condition, fp32)) != 0, self.shape)
          if not live.any():
            break
          self.run(s.subassignments, live, fp32)
      else:
        raise NotImplementedError(type(s).__name__)

  def init_temps(self, statements):
    for s in ot.walk_statements(statements):
      for root in ot.statement_exprs(s):
        for node in ot.walk_nodes(root):
          if isinstance(node, ot.TempVar) and id(node) not in self.temps:
            dt = node.datatype
            if dt == FP.BOOL:
              self.temps[id(node)] = np.zeros(self.shape, dtype=np.bool_)
            elif dt in (FP.INT, FP.UINT, FP.LONG, FP.ULONG):
              self.temps[id(node)] = np.zeros(self.shape, dtype=np.int64)
            else:
              self.temps[id(node)] = np.zeros(self.shape)


def evaluate_elementwise(descr, memory, elems, sym_names, tmp_values, fp32=False):
  """Run one ElementwiseDescr on the elements `elems`, updating memory / tmp_values.

  fp32=True rounds floating-point temporaries to float32 on assignment (the kernel's
  registers), which keeps comparisons against them consistent with an FP32 kernel;
  tensor values are stored unrounded either way.
  """
  st = _Stage(descr, memory, np.asarray(elems), sym_names, tmp_values)
  st.init_temps(descr.oplist)
  mask = np.ones(st.shape, dtype=np.bool_)
  st.run(descr.oplist, mask, fp32)
