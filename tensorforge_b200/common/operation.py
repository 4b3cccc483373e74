"""Operations of elementwise statements (tensorforge/common/operation.py:6-59).

The member names are the reference's. Unlike the reference, every member has its own
value: there the hyperbolic functions reuse the values of the circular ones
(SINH = 100 = SIN, ...), which makes them aliases, so `sinh(x)` would come out as
`sin(x)`. Here each name means the function it names.
"""
import enum


class Operation(enum.Enum):
  COPY = 0
  MIN = 1
  MAX = 2
  DIV = 3
  MUL = 4
  ADD = 5
  SUB = 6
  SQRT = 7
  POW = 8
  CBRT = 9
  MOD = 10
  NEG = 11
  RCP = 12
  RSQRT = 13
  RCBRT = 14
  ABS = 15
  CEIL = 30
  FLOOR = 31
  ROUND = 32
  SIGN = 33
  TRUNC = 34
  LOGP1 = 94
  EXPM1 = 95
  GAMMA = 96
  ERF = 97
  LOG = 98
  EXP = 99
  SIN = 100
  COS = 101
  TAN = 102
  ASIN = 103
  ACOS = 104
  ATAN = 105
  SINH = 110
  COSH = 111
  TANH = 112
  ASINH = 113
  ACOSH = 114
  ATANH = 115
  NOT = 1000
  AND = 1001
  OR = 1002
  XOR = 1003
  SHR = 1100
  SHL = 1101
  SHRS = 1102
  EQ = 2000
  NEQ = 2001
  LT = 2002
  LE = 2003
  GT = 2004
  GE = 2005


# one-argument floating-point functions: CUDA math library name (double form; the float
# form appends 'f')
UNARY_MATH = {
  Operation.SQRT: 'sqrt', Operation.CBRT: 'cbrt', Operation.RSQRT: 'rsqrt', Operation.RCBRT: 'rcbrt',
  Operation.ABS: 'fabs', Operation.CEIL: 'ceil', Operation.FLOOR: 'floor', Operation.ROUND: 'round',
  Operation.TRUNC: 'trunc', Operation.LOGP1: 'log1p', Operation.EXPM1: 'expm1', Operation.GAMMA: 'tgamma',
  Operation.ERF: 'erf', Operation.LOG: 'log', Operation.EXP: 'exp', Operation.SIN: 'sin', Operation.COS: 'cos',
  Operation.TAN: 'tan', Operation.ASIN: 'asin', Operation.ACOS: 'acos', Operation.ATAN: 'atan',
  Operation.SINH: 'sinh', Operation.COSH: 'cosh', Operation.TANH: 'tanh', Operation.ASINH: 'asinh',
  Operation.ACOSH: 'acosh', Operation.ATANH: 'atanh',
}

# two-argument floating-point functions
BINARY_MATH = {Operation.MIN: 'fmin', Operation.MAX: 'fmax', Operation.POW: 'pow', Operation.MOD: 'fmod'}

ARITHMETIC = {Operation.ADD: '+', Operation.SUB: '-', Operation.MUL: '*', Operation.DIV: '/'}

COMPARISON = {Operation.EQ: '==', Operation.NEQ: '!=', Operation.LT: '<', Operation.LE: '<=',
              Operation.GT: '>', Operation.GE: '>='}

# bitwise forms on integers; on booleans AND / OR / XOR / NOT are the logical ones
BITWISE = {Operation.AND: '&', Operation.OR: '|', Operation.XOR: '^', Operation.SHL: '<<',
           Operation.SHR: '>>', Operation.SHRS: '>>'}
LOGICAL = {Operation.AND: '&&', Operation.OR: '||', Operation.XOR: '!='}


def arity(op: Operation) -> int:
  if op in UNARY_MATH or op in (Operation.NEG, Operation.RCP, Operation.NOT, Operation.SIGN, Operation.COPY):
    return 1
  return 2
