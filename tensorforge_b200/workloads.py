"""Named descriptor chains: the benchmark workloads and the parity cases.

Every builder takes a namespace `ns` exposing the TensorForge frontend names (`Tensor`,
`SubTensor`, `BoundingBox`, `ListSPP`, `Addressing`, `MultilinearDescr`, `GemmDescr`,
`generate_tmp_tensor`), so the same chain can be built with the reference package and
with tensorforge_b200 and the two results compared on identical inputs. Builders only
describe inputs; they compute nothing. Shapes follow the reference's own test suites and
benchmark programs: tests/gemms/testsuites/*.yaml, benchmarks/fused/programs/s3time.cf,
benchmarks/simple-gemm/params.yaml.
"""
import numpy as np


def sparse_pattern(rows, cols, density, seed):
  """Seeded Bernoulli pattern, entries listed in column-major order."""
  rng = np.random.default_rng(seed)
  mask = rng.random((rows, cols)) < density
  return [(int(i), int(j)) for j in range(cols) for i in range(rows) if mask[i, j]]


def fixed_nnz_pattern(rows, cols, nnz, seed):
  """Seeded pattern with exactly `nnz` entries, column-major order."""
  rng = np.random.default_rng(seed)
  flat = np.sort(rng.choice(rows * cols, size=nnz, replace=False))
  ij = [(int(f % rows), int(f // rows)) for f in flat]
  return sorted(ij, key=lambda t: (t[1], t[0]))


def ns_from_module(root):
  """Namespace of frontend names from a package root ('tensorforge' or 'tensorforge_b200')."""
  import importlib
  tm = importlib.import_module(f'{root}.common.matrix.tensor')
  bb = importlib.import_module(f'{root}.common.matrix.boundingbox')
  sp = importlib.import_module(f'{root}.common.matrix.spp')
  bt = importlib.import_module(f'{root}.common.basic_types')
  de = importlib.import_module(f'{root}.generators.descriptions')
  ax = importlib.import_module(f'{root}.common.aux')

  class NS:
    pass
  ns = NS()
  ns.Tensor, ns.SubTensor = tm.Tensor, tm.SubTensor
  ns.BoundingBox = bb.BoundingBox
  ns.ListSPP, ns.MaskSPP, ns.FullSPP = sp.ListSPP, sp.MaskSPP, sp.FullSPP
  ns.Addressing = bt.Addressing
  ns.FloatingPointType = bt.FloatingPointType
  ns.MultilinearDescr, ns.GemmDescr = de.MultilinearDescr, de.GemmDescr
  ns.generate_tmp_tensor = ax.generate_tmp_tensor
  ns.ElementwiseDescr = de.ElementwiseDescr
  ns.optree = importlib.import_module(f'{root}.generators.optree')
  return ns


# --------------------------------------------------------------------------- chains

def plain_gemm(ns, m=56, k=56, n=9, addr_b='pointer_based', addr_c='pointer_based',
               addr_a='none', add=False, alpha=1.0):
  """C_e = A * B_e (BASELINE config 0 when m=k=56, n=9, B/C pointer arrays)."""
  A = ns.Tensor([m, k], ns.Addressing.str2addr(addr_a))
  B = ns.Tensor([k, n], ns.Addressing.str2addr(addr_b))
  C = ns.Tensor([m, n], ns.Addressing.str2addr(addr_c))
  if alpha != 1.0:
    return [ns.GemmDescr(False, False, ns.SubTensor(A), ns.SubTensor(B), ns.SubTensor(C), alpha=alpha)]
  return [ns.MultilinearDescr(ns.SubTensor(C), [ns.SubTensor(A), ns.SubTensor(B)],
                              [[0, -1], [-1, 1]], [[0, 1], [0, 1]], add=add)]


def volume_chain(ns, basis=56, quantities=9, terms=3, k_density=0.45, s_nnz=24, seed=0,
                 k_addr='none', q_addr='strided', s_addr='strided', out_addr='strided'):
  """out_e = sum_t K_t * Q_e * S_{e,t} (s3time.cf).

  K_t: shared sparse basis x basis (ListSPP, seeded Bernoulli(k_density) pattern).
  S_{e,t}: per-element sparse quantities x quantities with `s_nnz` seeded nonzeros,
  strided with the full q*q slot per element, values stored compactly at its start.
  """
  Q = ns.Tensor([basis, quantities], ns.Addressing.str2addr(q_addr))
  out = ns.Tensor([basis, quantities], ns.Addressing.str2addr(out_addr))
  descrs = []
  for t in range(terms):
    kp = sparse_pattern(basis, basis, k_density, seed * 1000 + 11 + t)
    sp = fixed_nnz_pattern(quantities, quantities, min(s_nnz, quantities * quantities), seed * 1000 + 101 + t)
    K = ns.Tensor([basis, basis], ns.Addressing.str2addr(k_addr),
                  spp=ns.ListSPP(kp, (basis, basis)) if k_density < 1.0 else None)
    S = ns.Tensor([quantities, quantities], ns.Addressing.str2addr(s_addr),
                  spp=ns.ListSPP(sp, (quantities, quantities)) if s_nnz < quantities * quantities else None)
    T = ns.generate_tmp_tensor([ns.SubTensor(K), ns.SubTensor(Q)], [[0, -1], [-1, 1]])
    descrs.append(ns.MultilinearDescr(ns.SubTensor(T), [ns.SubTensor(K), ns.SubTensor(Q)],
                                      [[0, -1], [-1, 1]], [[0, 1], [0, 1]]))
    descrs.append(ns.MultilinearDescr(ns.SubTensor(out), [ns.SubTensor(T), ns.SubTensor(S)],
                                      [[0, -1], [-1, 1]], [[0, 1], [0, 1]], add=(t > 0)))
  return descrs


def subbox_gemm(ns, box_a, box_b, box_c, shape=56, addr='strided', trans_a=False, trans_b=False):
  """Sub-bounding-box GEMMs from tests/gemms/testsuites/notrans-notrans-tests.yaml:1-35."""
  BB = ns.BoundingBox
  A = ns.Tensor([shape, shape], ns.Addressing.str2addr(addr), BB(box_a[:2], box_a[2:]))
  B = ns.Tensor([shape, shape], ns.Addressing.str2addr(addr), BB(box_b[:2], box_b[2:]))
  C = ns.Tensor([shape, shape], ns.Addressing.str2addr(addr), BB(box_c[:2], box_c[2:]))
  return [ns.GemmDescr(trans_a, trans_b, ns.SubTensor(A), ns.SubTensor(B), ns.SubTensor(C))]


def suite_gemm(ns, a, b, c, trans_a=False, trans_b=False, alpha=1.0):
  """One GEMM of the reference's YAML test suites (tests/gemms/testsuites/*.yaml): each of
  a, b, c is {'rows', 'cols', 'addressing', 'bbox': [r0, c0, r1, c1]} in stored order."""
  BB = ns.BoundingBox

  def tensor(m):
    box = m['bbox']
    return ns.Tensor([m['rows'], m['cols']], ns.Addressing.str2addr(m['addressing']), BB(box[:2], box[2:]))
  A, B, C = tensor(a), tensor(b), tensor(c)
  return [ns.GemmDescr(trans_a, trans_b, ns.SubTensor(A), ns.SubTensor(B), ns.SubTensor(C), alpha=alpha)]


def three_matrices(ns):
  """D += A x (B x C) with a temporary (example/three_matrices.py:9-32)."""
  BB = ns.BoundingBox
  D = ns.Tensor([56, 9], ns.Addressing.STRIDED, BB([0, 0], [56, 9]))
  A = ns.Tensor([56, 56], ns.Addressing.STRIDED, BB([0, 0], [56, 56]))
  B = ns.Tensor([56, 9], ns.Addressing.STRIDED, BB([0, 0], [56, 9]))
  C = ns.Tensor([9, 9], ns.Addressing.STRIDED, BB([0, 0], [9, 9]))
  T = ns.generate_tmp_tensor([ns.SubTensor(B), ns.SubTensor(C)], [[0, -1], [-1, 1]])
  return [ns.MultilinearDescr(ns.SubTensor(T), [ns.SubTensor(B), ns.SubTensor(C)], [[0, -1], [-1, 1]], [[0, 1], [0, 1]]),
          ns.MultilinearDescr(ns.SubTensor(D), [ns.SubTensor(A), ns.SubTensor(T)], [[0, -1], [-1, 1]], [[0, 1], [0, 1]], add=True)]


def sparse_dense(ns, m=20, k=20, n=9, density=0.3, seed=5, sparse_side='a', addr_sparse='none'):
  """Sparse x dense and dense x sparse GEMMs (tests/{sparse_dense,dense_sparse}_gemms)."""
  if sparse_side == 'a':
    pat = sparse_pattern(m, k, density, seed)
    A = ns.Tensor([m, k], ns.Addressing.str2addr(addr_sparse), spp=ns.ListSPP(pat, (m, k)))
    B = ns.Tensor([k, n], ns.Addressing.STRIDED)
  else:
    pat = sparse_pattern(k, n, density, seed)
    A = ns.Tensor([m, k], ns.Addressing.NONE)
    B = ns.Tensor([k, n], ns.Addressing.str2addr(addr_sparse), spp=ns.ListSPP(pat, (k, n)))
  C = ns.Tensor([m, n], ns.Addressing.STRIDED)
  return [ns.MultilinearDescr(ns.SubTensor(C), [ns.SubTensor(A), ns.SubTensor(B)], [[0, -1], [-1, 1]], [[0, 1], [0, 1]])]


def rank3(ns):
  """dest[i,j,l] = sum_k A[i,k] * B[k,j,l] (a general multilinear product)."""
  A = ns.Tensor([10, 6], ns.Addressing.NONE)
  B = ns.Tensor([6, 5, 4], ns.Addressing.STRIDED)
  D = ns.Tensor([10, 5, 4], ns.Addressing.STRIDED)
  return [ns.MultilinearDescr(ns.SubTensor(D), [ns.SubTensor(A), ns.SubTensor(B)],
                              [[0, -1], [-1, 1, 2]], [[0, 1], [0, 1, 2]])]


def two_contractions(ns):
  """dest[i,j] = sum_{k,l} A[i,k,l] * B[k,l,j] (two contracted indices)."""
  A = ns.Tensor([8, 4, 3], ns.Addressing.NONE)
  B = ns.Tensor([4, 3, 7], ns.Addressing.PTR_BASED)
  D = ns.Tensor([8, 7], ns.Addressing.PTR_BASED)
  return [ns.MultilinearDescr(ns.SubTensor(D), [ns.SubTensor(A), ns.SubTensor(B)],
                              [[0, -1, -2], [-1, -2, 1]], [[0, 1, 2], [0, 1, 2]])]


def scalar_scaled(ns):
  """dest[i,j] = A[i,k] * B[k,j] * s with a SCALAR operand passed by value."""
  A = ns.Tensor([16, 12], ns.Addressing.NONE)
  B = ns.Tensor([12, 5], ns.Addressing.STRIDED)
  S = ns.Tensor([], ns.Addressing.SCALAR)
  D = ns.Tensor([16, 5], ns.Addressing.STRIDED)
  return [ns.MultilinearDescr(ns.SubTensor(D), [ns.SubTensor(A), ns.SubTensor(B), ns.SubTensor(S)],
                              [[0, -1], [-1, 1], []], [[0, 1], [0, 1], []])]


def outer_product(ns):
  """dest[i,j] = a[i] * b[j] (no contraction)."""
  a = ns.Tensor([13], ns.Addressing.STRIDED)
  b = ns.Tensor([7], ns.Addressing.NONE)
  D = ns.Tensor([13, 7], ns.Addressing.STRIDED)
  return [ns.MultilinearDescr(ns.SubTensor(D), [ns.SubTensor(a), ns.SubTensor(b)], [[0], [1]], [[0], [0]])]


def kat_matmul(ns, trans_a=False, trans_b=False, size=32):
  """The yateto code-generation matmul fixtures (tests/code-gen/matmul/ssm_86_Eigen:
  kernel.cpp:9-60, subroutine.h:3-6): C = op(A) op(B) for 32x32 pointer-array operands,
  written as the descriptor lists whose launchers have the fixtures' parameter order --
  (C, A, B) for AB; (A, B, C) for A^T B, where yateto forms the product into a temporary
  that is then copied to C; (A, C, B) for A B^T and A^T B^T, where A (transposed or not) is
  first copied into a temporary."""
  P = ns.Addressing.PTR_BASED
  A, B, C = ns.Tensor([size, size], P), ns.Tensor([size, size], P), ns.Tensor([size, size], P)
  ident = [[0, 1], [0, 1]]
  sub = ns.SubTensor
  if not trans_a and not trans_b:
    return [ns.MultilinearDescr(sub(C), [sub(A), sub(B)], [[0, -1], [-1, 1]], ident)]
  T = ns.Tensor([size, size], ns.Addressing.STRIDED, is_tmp=True)
  if trans_a and not trans_b:
    return [ns.MultilinearDescr(sub(T), [sub(A), sub(B)], [[-1, 0], [-1, 1]], ident),
            ns.MultilinearDescr(sub(C), [sub(T)], [[0, 1]], [[0, 1]])]
  copy = [[1, 0]] if trans_a else [[0, 1]]
  return [ns.MultilinearDescr(sub(T), [sub(A)], copy, [[0, 1]]),
          ns.MultilinearDescr(sub(C), [sub(T), sub(B)], [[0, -1], [1, -1]], ident)]


CASES = {
  # name: (builder, kwargs, num_elements)
  'c0_gemm_ptr': (plain_gemm, {}, 24),
  'c0_gemm_strided': (plain_gemm, {'addr_b': 'strided', 'addr_c': 'strided'}, 16),
  'gemm_add': (plain_gemm, {'m': 24, 'k': 17, 'n': 5, 'addr_b': 'strided', 'addr_c': 'strided', 'add': True}, 16),
  'gemm_alpha': (plain_gemm, {'m': 12, 'k': 8, 'n': 4, 'addr_b': 'strided', 'addr_c': 'strided', 'alpha': 1.5}, 8),
  'gemm_batched_a': (plain_gemm, {'m': 33, 'k': 9, 'n': 11, 'addr_a': 'strided', 'addr_b': 'strided', 'addr_c': 'strided'}, 16),
  'chain_o6': (volume_chain, {}, 16),
  'chain_o4_q27': (volume_chain, {'basis': 20, 'quantities': 27, 's_nnz': 72, 'seed': 3}, 16),
  'chain_o3_dense': (volume_chain, {'basis': 10, 'quantities': 9, 'k_density': 1.0, 's_nnz': 81, 'seed': 1, 'terms': 2}, 16),
  'chain_o6_ptr': (volume_chain, {'q_addr': 'pointer_based', 's_addr': 'pointer_based', 'out_addr': 'pointer_based'}, 16),
  'subbox_0': (subbox_gemm, {'box_a': [0, 0, 33, 9], 'box_b': [0, 0, 9, 11], 'box_c': [0, 0, 33, 11]}, 3),
  'subbox_1': (subbox_gemm, {'box_a': [22, 46, 55, 55], 'box_b': [46, 44, 55, 55], 'box_c': [0, 44, 33, 55]}, 3),
  'subbox_2': (subbox_gemm, {'box_a': [11, 23, 44, 32], 'box_b': [23, 22, 32, 33], 'box_c': [11, 22, 44, 33]}, 3),
  'trans_a': (subbox_gemm, {'box_a': [0, 0, 20, 20], 'box_b': [0, 0, 20, 7], 'box_c': [0, 0, 20, 7], 'shape': 20, 'trans_a': True}, 8),
  'three_matrices': (three_matrices, {}, 5),
  'sparse_a_shared': (sparse_dense, {'sparse_side': 'a'}, 16),
  'sparse_a_batched': (sparse_dense, {'sparse_side': 'a', 'addr_sparse': 'strided'}, 16),
  'sparse_b_batched': (sparse_dense, {'sparse_side': 'b', 'addr_sparse': 'strided'}, 16),
  'rank3': (rank3, {}, 8),
  'two_contractions': (two_contractions, {}, 8),
  'scalar_scaled': (scalar_scaled, {}, 8),
  'outer_product': (outer_product, {}, 8),
  'kat_matmul_ab': (kat_matmul, {}, 1),
  'kat_matmul_atb': (kat_matmul, {'trans_a': True}, 1),
  'kat_matmul_abt': (kat_matmul, {'trans_b': True}, 1),
  'kat_matmul_atbt': (kat_matmul, {'trans_a': True, 'trans_b': True}, 1),
}


def build(name, ns):
  """Descriptor list of a named case; `mixed_<basis>_<quantities>` names one group of the
  mixed-shape workload (`mixed_chain`)."""
  if name.startswith('mixed_') and name not in CASES:
    _, b, q = name.split('_')
    return mixed_chain(ns, int(b), int(q))
  fn, kwargs, _ = CASES[name]
  return fn(ns, **kwargs)


def num_elements(name):
  return CASES[name][2]


MIXED_BASES = (10, 20, 35, 56, 84)
MIXED_QUANTITIES = (9, 27)


def mixed_shape_groups(total=1_500_000, seed=0, lo=1_000, hi=200_000):
  """basis sizes {10,20,35,56,84} x quantity counts {9,27}.

  Returns [(basis, quantities, element count)], counts drawn log-uniform over lo..hi from
  `seed`, rescaled to sum to ~`total`, each rounded to a multiple of 8.
  """
  rng = np.random.default_rng(seed)
  shapes = [(b, q) for b in MIXED_BASES for q in MIXED_QUANTITIES]
  raw = np.exp(rng.uniform(np.log(lo), np.log(hi), len(shapes)))
  raw = raw * (total / raw.sum())
  counts = [max(8, int(round(c / 8)) * 8) for c in raw]
  return [(b, q, c) for (b, q), c in zip(shapes, counts)]


def mixed_chain(ns, basis, quantities, seed=0):
  """The order-`basis` volume chain with patterns seeded per shape (S density ~30%)."""
  nnz = max(1, int(round(0.3 * quantities * quantities)))
  return volume_chain(ns, basis=basis, quantities=quantities, s_nnz=nnz, seed=seed * 100 + basis * 7 + quantities)


# --------------------------------------------------------------------------- elementwise
# Statement programs over batched tensors (`ElementwiseDescr`), alone and fused with
# contractions. Built with tensorforge_b200 only: the reference's optree binds tensor
# variables through yateto, and its code generators do not emit elementwise stages.

def ew_update(ns, rows=56, cols=9, addr='strided'):
  """Pointwise nonlinear update of one 56x9 block per element, with a scalar gain:

      t = Q * s;  O = t > 0 ? t * exp(-t * t) : 0.5 * t

  One read and one write of the block: the HBM-bound elementwise workload."""
  ot = ns.optree
  a = ns.Addressing.str2addr(addr)
  Q, O = ns.Tensor([rows, cols], a), ns.Tensor([rows, cols], a)
  s = ns.Tensor([], ns.Addressing.SCALAR)
  t = ot.temp()
  return [ns.ElementwiseDescr([
    ot.assign(t, ot.tensor(Q) * ot.scalar(s)),
    ot.assign(ot.tensor(O), ot.ternary(t > 0.0, t * ot.exp(-(t * t)), 0.5 * t)),
  ])]


EW_FUNCTIONS = [
  # (name, expression builder over x in [-1, 1]) -- arguments kept inside each domain
  ('exp', lambda ot, x: ot.exp(x)), ('log', lambda ot, x: ot.log(ot.abs(x) + 0.5)),
  ('expm1', lambda ot, x: ot.expm1(x)), ('logp1', lambda ot, x: ot.logp1(ot.abs(x))),
  ('sqrt', lambda ot, x: ot.sqrt(ot.abs(x))), ('cbrt', lambda ot, x: ot.cbrt(x)),
  ('rsqrt', lambda ot, x: ot.rsqrt(ot.abs(x) + 0.25)),
  ('rcbrt', lambda ot, x: ot.rcbrt(x + 2.0)), ('pow', lambda ot, x: ot.pow(ot.abs(x) + 0.5, 1.3)),
  ('sin', lambda ot, x: ot.sin(3.0 * x)), ('cos', lambda ot, x: ot.cos(3.0 * x)),
  ('tan', lambda ot, x: ot.tan(x)), ('asin', lambda ot, x: ot.asin(0.9 * x)),
  ('acos', lambda ot, x: ot.acos(0.9 * x)), ('atan', lambda ot, x: ot.atan(4.0 * x)),
  ('sinh', lambda ot, x: ot.sinh(2.0 * x)), ('cosh', lambda ot, x: ot.cosh(2.0 * x)),
  ('tanh', lambda ot, x: ot.tanh(2.0 * x)), ('asinh', lambda ot, x: ot.asinh(3.0 * x)),
  ('acosh', lambda ot, x: ot.acosh(ot.abs(x) + 1.5)), ('atanh', lambda ot, x: ot.atanh(0.9 * x)),
  ('erf', lambda ot, x: ot.erf(2.0 * x)), ('gamma', lambda ot, x: ot.gamma(x + 2.0)),
  ('abs', lambda ot, x: abs(x)), ('neg', lambda ot, x: -x), ('rcp', lambda ot, x: 1.0 / (x + 2.0)),
  ('ceil', lambda ot, x: ot.ceil(4.0 * x)), ('floor', lambda ot, x: ot.floor(4.0 * x)),
  ('round', lambda ot, x: ot.round(4.0 * x)), ('trunc', lambda ot, x: ot.trunc(4.0 * x)),
  ('sign', lambda ot, x: ot.sign(x)), ('mod', lambda ot, x: (8.0 * x) % 3.0),
  ('min', lambda ot, x: ot.min(x, 0.25)), ('max', lambda ot, x: ot.max(x, -0.25)),
  ('square', lambda ot, x: x ** 2), ('div', lambda ot, x: x / (x * x + 1.0)),
]


def ew_functions(ns, rows=12, cols=5):
  """One stage per operation, each writing its own slice O[:, :, f] of a rank-3 output
  (a view with a nonzero box corner in the last dimension)."""
  ot = ns.optree
  Q = ns.Tensor([rows, cols], ns.Addressing.STRIDED)
  O = ns.Tensor([rows, cols, len(EW_FUNCTIONS)], ns.Addressing.STRIDED)
  out = []
  for f, (_, fn) in enumerate(EW_FUNCTIONS):
    view = ns.SubTensor(O, ns.BoundingBox([0, 0, f], [rows, cols, f + 1]))
    out.append(ns.ElementwiseDescr([ot.assign(ot.tensor(view), fn(ot, ot.tensor(Q)))]))
  return out


def ew_control(ns, rows=20, cols=7):
  """Temporaries, if, ternary, a while loop with an integer counter, casts and integer /
  boolean operators: Newton's iteration for sqrt(x^2 + 1) plus branch-dependent terms."""
  ot = ns.optree
  FP = ns.FloatingPointType
  Q = ns.Tensor([rows, cols], ns.Addressing.PTR_BASED)
  P = ns.Tensor([rows, cols], ns.Addressing.STRIDED)
  O = ns.Tensor([rows, cols], ns.Addressing.STRIDED)
  x, y, i, flag = ot.temp(), ot.temp(), ot.temp(FP.INT), ot.temp(FP.BOOL)
  q, p, o = ot.tensor(Q), ot.tensor(P), ot.tensor(O)
  return [ns.ElementwiseDescr([
    ot.assign(x, q * q + 1.0),
    ot.assign(y, x),
    ot.loop(i < 6, [ot.assign(y, 0.5 * (y + x / y)), ot.assign(i, i + 1)]),
    ot.assign(flag, (q > 0.0) & ~(p < -0.5)),
    ot.assign(o, y),
    ot.conditional(flag, [ot.assign(o, o + p)]),
    ot.conditional((q < 0.0) | (p > 0.5), [ot.assign(o, o - ot.cast(ot.cast(4.0 * p, FP.INT) % 3, FP.FLOAT) * 0.125)]),
    ot.assign(o, o + ot.ternary(ot.bitxor(q > 0.0, p > 0.0), 2.0, ot.cast(i & 3, FP.FLOAT))),
  ])]


def ew_fused_chain(ns, basis=20, quantities=9):
  """A contraction into a temporary followed by an elementwise stage that accumulates a
  rectified copy into the output: T = K * Q;  O = O + max(T, 0) * s."""
  ot = ns.optree
  K = ns.Tensor([basis, basis], ns.Addressing.NONE)
  Q = ns.Tensor([basis, quantities], ns.Addressing.STRIDED)
  O = ns.Tensor([basis, quantities], ns.Addressing.PTR_BASED)
  s = ns.Tensor([], ns.Addressing.SCALAR)
  T = ns.generate_tmp_tensor([ns.SubTensor(K), ns.SubTensor(Q)], [[0, -1], [-1, 1]])
  o = ot.tensor(O)
  return [
    ns.MultilinearDescr(ns.SubTensor(T), [ns.SubTensor(K), ns.SubTensor(Q)], [[0, -1], [-1, 1]], [[0, 1], [0, 1]]),
    ns.ElementwiseDescr([ot.assign(o, o + ot.max(ot.tensor(T), 0.0) * ot.scalar(s))]),
  ]


def ew_feeds_contraction(ns, basis=16, quantities=9):
  """An elementwise stage defines a temporary that a contraction consumes:
  T = tanh(Q);  O = K * T;  O = O * O."""
  ot = ns.optree
  K = ns.Tensor([basis, basis], ns.Addressing.NONE)
  Q = ns.Tensor([basis, quantities], ns.Addressing.STRIDED)
  O = ns.Tensor([basis, quantities], ns.Addressing.STRIDED)
  T = ns.Tensor([basis, quantities], ns.Addressing.STRIDED, is_tmp=True)
  return [
    ns.ElementwiseDescr([ot.assign(ot.tensor(T), ot.tanh(ot.tensor(Q)))]),
    ns.MultilinearDescr(ns.SubTensor(O), [ns.SubTensor(K), ns.SubTensor(T)], [[0, -1], [-1, 1]], [[0, 1], [0, 1]]),
    ns.ElementwiseDescr([ot.assign(ot.tensor(O), ot.tensor(O) ** 2)]),
  ]


def ew_views(ns):
  """Sub-box views and a transposed read: O[2+n0, 1+n1] = Q[3+n1, 4+n0] * 2 + B[n0, n1]
  with a 6x5 index box."""
  ot = ns.optree
  Q = ns.Tensor([10, 12], ns.Addressing.STRIDED)
  B = ns.Tensor([6, 5], ns.Addressing.NONE)
  O = ns.Tensor([9, 8], ns.Addressing.STRIDED)
  qv = ns.SubTensor(Q, ns.BoundingBox([3, 4], [8, 10]))
  ov = ns.SubTensor(O, ns.BoundingBox([2, 1], [8, 6]))
  return [ns.ElementwiseDescr([
    ot.assign(ot.tensor(ov), ot.tensor(qv, indices=[-2, -1]) * 2.0 + ot.tensor(B)),
  ])]


def ew_sparse_read(ns, rows=14, cols=9, seed=4):
  """A compactly stored sparse operand read pointwise (absent entries read 0):
  O = 2 * S + 1."""
  ot = ns.optree
  S = ns.Tensor([rows, cols], ns.Addressing.STRIDED, spp=ns.ListSPP(sparse_pattern(rows, cols, 0.4, seed), [rows, cols]))
  O = ns.Tensor([rows, cols], ns.Addressing.STRIDED)
  return [ns.ElementwiseDescr([ot.assign(ot.tensor(O), 2.0 * ot.tensor(S) + 1.0)])]


def ew_chain_epilogue(ns, basis=56, quantities=9, terms=3, seed=0, accumulate=False):
  """The volume chain followed by a pointwise update of its output, fused as an epilogue of
  the column program:  out = sum_t K_t Q S_t (+ out);  out = out > 0 ? out : 0.1 * out;
  out = out + P * s  (P a second per-element 56x9 input, s a scalar)."""
  ot = ns.optree
  descrs = volume_chain(ns, basis=basis, quantities=quantities, terms=terms, seed=seed)
  out = descrs[-1].dest.tensor
  if accumulate:
    descrs[1].add = True
  P = ns.Tensor([basis, quantities], ns.Addressing.STRIDED)
  s = ns.Tensor([], ns.Addressing.SCALAR)
  o = ot.tensor(out)
  descrs.append(ns.ElementwiseDescr([
    ot.assign(o, ot.ternary(o > 0.0, o, 0.1 * o)),
    ot.assign(o, o + ot.tensor(P) * ot.scalar(s)),
  ]))
  return descrs


EW_CASES = {
  # name: (builder, kwargs, num_elements)
  'ew_update': (ew_update, {}, 37),
  'ew_functions': (ew_functions, {}, 9),
  'ew_control': (ew_control, {}, 21),
  'ew_fused_chain': (ew_fused_chain, {}, 19),
  'ew_feeds_contraction': (ew_feeds_contraction, {}, 11),
  'ew_views': (ew_views, {}, 7),
  'ew_sparse_read': (ew_sparse_read, {}, 13),
  'ew_chain_epilogue': (ew_chain_epilogue, {}, 29),
  'ew_chain_epilogue_add': (ew_chain_epilogue, {'basis': 20, 'quantities': 9, 'accumulate': True, 'seed': 2}, 23),
}


def build_elementwise(name, ns):
  fn, kwargs, _ = EW_CASES[name]
  return fn(ns, **kwargs)
