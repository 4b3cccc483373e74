"""FP64 tensor-core generator (DMMA, `mma.sync.m8n8k4.f64`) for shared-left GEMM chains.

Computes out_e (+)= sum_t A_t * (B_{e,t} * R_{e,t}) (plan/chains.py) for FP64 operands.
tcgen05 has no FP64 kind, so the FP64 tensor-core instruction on sm_100a is the warp-level
DMMA. One CTA walks tiles of TE whole elements (C = TE*N flat output columns (e, j), C a
multiple of 8):

  1. U phase (CUDA cores): one thread per (element, row l) reads row l of B_{e,t} with
     coalesced loads and writes row l of U_t = B_{e,t} * R_{e,t} (R's compile-time pattern
     unrolled) into shared memory, column-major per flat column: U_t[c][k], pitch LD.
  2. MMA phase: warp w owns the 8-row block mb = w % MB of the output and the 8-column
     blocks nb = w / MB + NS*i; for every term and every 4-wide k step it loads one A
     fragment (A_t densified and zero-padded in shared memory, staged once per CTA) and,
     per owned column block, one U fragment, and issues m8n8k4 DMMAs into FP64
     accumulators that persist across terms.
  3. Epilogue: the accumulators are staged in shared memory (pitch LDO) and written back
     with coalesced stores (accumulated into out_e when the chain adds, skipped for
     elements whose flag is 0).

With plan option prefetch=1 (the default when it fits in shared memory) the next tile's
batched B and R values are copied into a stage with cp.async right after the U phase has
consumed it, so the loads overlap the MMA phase and the epilogue.

Pitches: LD = 4 (mod 8) doubles makes both fragment loads (lane -> row lane/4, k lane%4)
bank-conflict free; LDO = 2 (mod 4) does the same for the epilogue's fragment stores.
Padded k rows of U and A stay zero, so K need not be a multiple of 4. The contraction
order (A_t * (B * R_t)) matches the column-program generator; results agree with the
reference order within FP64 rounding.
"""
from math import gcd

from ..plan.chains import match_left_chain

DMMA_HELPERS = r'''
#ifndef TFB_DMMA_HELPERS
#define TFB_DMMA_HELPERS
namespace tfb_dmma {
// D = A * B + D for one m8n8k4 FP64 tile: a = A[lane/4][lane%4], b = B[lane%4][lane/4],
// d = D[lane/4][2*(lane%4) + {0,1}]
__device__ __forceinline__ void mma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}
}  // namespace tfb_dmma
#endif
'''


def _pad(x, m):
  return (x + m - 1) // m * m


def staged_ops(shape):
  """Distinct batched operands a tile reads: [(operand, values per element)], B before R."""
  out = []
  for role in ('B', 'R'):
    for t in shape.terms:
      op = getattr(t, role)
      if op is None or op.kind != 'batched' or any(op is o for o, _ in out):
        continue
      out.append((op, op.storage_size() if op.sparse else op.element_volume()))
  return out


def layout(shape, te, prefetch=False):
  """Pitches and shared-memory regions (in doubles) for a tile of `te` elements.

  With prefetch, the next tile's batched B and R values are copied with cp.async into a
  stage region while the current tile's MMAs run; R is then read from the stage.
  """
  M, N = shape.M, shape.N
  kp = _pad(max(t.K for t in shape.terms), 4)
  ld = kp if kp % 8 == 4 else kp + 4
  mp = _pad(M, 8)
  ldo = M + ((2 - M) % 4)
  C = te * N
  nterms = len(shape.terms)
  a_vals = nterms * mp * ld
  u_vals = nterms * C * ld
  o_vals = C * ldo
  r_vals = 0
  r_off = {}
  for t in shape.terms:
    if t.R is not None and t.R.kind == 'batched' and t.R.name not in r_off:
      r_off[t.R.name] = r_vals
      r_vals += te * _pad(t.R.storage_size(), 2)
  region = max(u_vals, o_vals)
  stage_off, stage = {}, 0
  if prefetch:
    r_vals, r_off = 0, {}
    for op, vals in staged_ops(shape):
      stage_off[op.name] = stage
      stage += te * _pad(vals, 2)
  return dict(KP=kp, LD=ld, MP=mp, LDO=ldo, C=C, A=a_vals, U=u_vals, O=o_vals, R=r_vals, r_off=r_off,
              region=region, stage=stage, stage_off=stage_off, prefetch=prefetch,
              total=a_vals + region + r_vals + stage)


def plan(chain, shape, variant, smem_limit):
  """Tile size and warp split, or None if the chain does not fit."""
  from ..plan import Plan
  M, N = shape.M, shape.N
  if M > 128 or N > 64 or max(t.K for t in shape.terms) > 128:
    return None
  te0 = 8 // gcd(N, 8)
  target = variant.get('columns', 72)
  te_max = variant.get('tile_elements') or max(te0, (target // N) // te0 * te0)
  lay = None
  for prefetch in ((1, 0) if variant.get('prefetch', 1) else (0,)):
    te = te_max
    while te >= te0:
      lay = layout(shape, te, bool(prefetch))
      if lay['total'] * 8 <= smem_limit:
        break
      te -= te0
    if te >= te0:
      break
  else:
    return None
  mb = lay['MP'] // 8
  nb = lay['C'] // 8
  # column blocks are split evenly over warp groups: the most warps (at most 32 per CTA)
  # that still leave every warp two or more independent accumulator chains (measured on
  # the order-6 chain: 3 groups of 7 warps 1.29e8 el/s, 2 groups 1.19e8, 4 groups 1.16e8)
  ns = variant.get('nsplit')
  if not ns:
    fits = [d for d in range(1, nb + 1) if nb % d == 0 and mb * d <= 32]
    ns = max([d for d in fits if nb // d >= 2] or fits or [1])
  ns = max(1, min(ns, nb, 1024 // (32 * mb)))
  threads = 32 * mb * ns
  if threads > 1024:
    return None
  return Plan('dmma', {'tile_elements': te, 'nsplit': ns, 'prefetch': prefetch}, lay['total'] * 8, threads,
              note=f'M={M} N={N} terms={len(shape.terms)} C={lay["C"]} warps={mb * ns}')


def emit_dmma(chain, plan_, context, base_name, globals_):
  shape = match_left_chain(chain)
  return _Dmma(chain, shape, plan_, context, base_name).emit(globals_)


class _Dmma:
  def __init__(self, chain, shape, plan_, ctx, base):
    assert ctx.fp_as_str() == 'double'
    self.chain, self.s, self.plan, self.ctx, self.base = chain, shape, plan_, ctx, base
    self.TE = plan_.params['tile_elements']
    self.NS = plan_.params['nsplit']
    self.L = layout(shape, self.TE, bool(plan_.params.get('prefetch', 0)))
    self.MB = self.L['MP'] // 8
    self.NB = self.L['C'] // 8
    self.BT = 32 * self.MB * self.NS
    self.lines = []
    self.ind = 0

  def w(self, s=''):
    self.lines.append('  ' * self.ind + s)

  def open(self, head):
    self.w(head + ' {')
    self.ind += 1

  def close(self):
    self.ind -= 1
    self.w('}')

  def params(self, globals_):
    out = []
    for t, _ in globals_:
      dt = 'double' if t.datatype is None else str(t.datatype)
      if t.addressing.name == 'SCALAR':
        out.append(f'{dt} {t.name}')
      else:
        const = 'const ' if t.direction.name == 'SOURCE' else ''
        out.append(f'{const}{dt}{t.addressing.to_pointer()} __restrict__ {t.name}')
        if t.addressing.name != 'NONE':
          out.append(f'unsigned {t.name}_extraOffset')
    return out + ['size_t numElements', 'const unsigned* __restrict__ flags']

  def _elem_ptr(self, op, e):
    a = op.addressing.name
    if a == 'STRIDED':
      return f'({op.name} + ({e}) * {op.element_volume()}u + {op.name}_extraOffset)'
    if a == 'PTR_BASED':
      return f'({op.name}[{e}] + {op.name}_extraOffset)'
    return op.name

  # ------------------------------------------------------------------ pieces
  def _a_tables(self):
    """Shared-memory slot (row * LD + k) of every stored value of each sparse A_t."""
    b, L = self.base, self.L
    for ti, t in enumerate(self.s.terms):
      if t.A.sparse:
        slots = [0] * t.A.storage_size()
        for (i, k), pos in t.A.sparse_lookup().items():
          slots[pos] = i * L['LD'] + k
        self.w(f'__device__ const unsigned dmma_aslot_{b}_{ti}[{len(slots)}] = {{{", ".join(map(str, slots))}}};')

  def _stage_a(self):
    s, L, BT, b = self.s, self.L, self.BT, self.base
    self.w(f'for (unsigned q = threadIdx.x; q < {L["A"] + L["U"]}u; q += {BT}u) smem[q] = 0.0;')
    self.w('__syncthreads();')
    for ti, t in enumerate(s.terms):
      base = ti * L['MP'] * L['LD']
      n = t.A.storage_size()
      if t.A.sparse:
        self.w(f'for (unsigned q = threadIdx.x; q < {n}u; q += {BT}u) '
               f'sA[{base} + dmma_aslot_{b}_{ti}[q]] = {t.A.name}[q];')
      else:
        M = s.M
        self.w(f'for (unsigned q = threadIdx.x; q < {n}u; q += {BT}u) '
               f'sA[{base} + (q % {M}u) * {L["LD"]}u + q / {M}u] = {t.A.name}[q];')
    self.w('__syncthreads();')

  def _stage_r(self):
    L, BT, TE = self.L, self.BT, self.TE
    ops = {o.name: o for o in self.chain.operands}
    for name, off in L['r_off'].items():
      op = ops[name]
      nr = op.storage_size()
      nrp = _pad(nr, 2)
      self.open(f'for (unsigned q = threadIdx.x; q < {TE * nr}u; q += {BT}u)')
      self.w(f'const unsigned ei = q / {nr}u, p = q - ei * {nr}u;')
      self.w('const size_t e = e0 + ei;')
      self.w('const bool live = e < numElements && (flags == nullptr || flags[e] != 0u);')
      self.w(f'sR[{off} + ei * {nrp}u + p] = live ? __ldg({self._elem_ptr(op, "e")} + p) : 0.0;')
      self.close()

  def _prefetch(self, tile_expr):
    """cp.async the tile's batched B / R values into the stage (16-byte chunks when aligned)."""
    L, BT, TE = self.L, self.BT, self.TE
    for op, vals in staged_ops(self.s):
      off = L['stage_off'][op.name]
      vp = _pad(vals, 2)
      self.open('')
      self.w(f'const size_t pe0 = ({tile_expr}) * {TE}u;')
      pairs = vals // 2
      if pairs:
        self.open(f'for (unsigned q = threadIdx.x; q < {TE * pairs}u; q += {BT}u)')
        self.w(f'const unsigned ei = q / {pairs}u, c2 = q - ei * {pairs}u;')
        self.w('const size_t ee = pe0 + ei;')
        self.open('if (ee < numElements && (flags == nullptr || flags[ee] != 0u))')
        self.w(f'const double* src = {self._elem_ptr(op, "ee")} + 2u * c2;')
        self.w(f'double* dst = sS + {off}u + ei * {vp}u + 2u * c2;')
        self.w('if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0u) tfb_cp::copy16(dst, src);')
        self.w('else { tfb_cp::copy8(dst, src); tfb_cp::copy8(dst + 1, src + 1); }')
        self.close()
        self.close()
      if vals % 2:
        self.open(f'for (unsigned ei = threadIdx.x; ei < {TE}u; ei += {BT}u)')
        self.w('const size_t ee = pe0 + ei;')
        self.w(f'if (ee < numElements && (flags == nullptr || flags[ee] != 0u)) '
               f'tfb_cp::copy8(sS + {off}u + ei * {vp}u + {vals - 1}u, {self._elem_ptr(op, "ee")} + {vals - 1}u);')
        self.close()
      self.close()

  def _u_phase(self):
    """U_t[c][l] = sum_m B_t[l][m] * R_t[m][j] for c = e*N + j; terms sharing B load it once."""
    s, L, BT, TE = self.s, self.L, self.BT, self.TE
    N, LD, C = s.N, L['LD'], L['C']
    groups = {}
    for ti, t in enumerate(s.terms):
      groups.setdefault(t.B.name, []).append((ti, t))
    for bname, terms in groups.items():
      B = terms[0][1].B
      K, P = terms[0][1].K, terms[0][1].P
      KP = _pad(K, 4)
      # rows K..KP-1 are written as zeros: the epilogue reuses this region as its stage
      self.open(f'for (unsigned q = threadIdx.x; q < {TE * KP}u; q += {BT}u)')
      self.w(f'const unsigned ei = q / {KP}u, l = q - ei * {KP}u;')
      self.w('const size_t e = e0 + ei;')
      self.w(f'const bool live = l < {K}u && e < numElements && (flags == nullptr || flags[e] != 0u);')
      if L['prefetch']:
        bvp = _pad(B.element_volume(), 2)
        self.w(f'const double* const bq = sS + {L["stage_off"][B.name]}u + ei * {bvp}u + (live ? l : 0u);')
        for m in range(P):
          self.w(f'const double q{m} = live ? bq[{m * K}u] : 0.0;')
      else:
        self.w(f'const double* const bq = live ? {self._elem_ptr(B, "e")} + l : nullptr;')
        for m in range(P):
          self.w(f'const double q{m} = live ? __ldg(bq + {m * K}u) : 0.0;')
      for ti, t in terms:
        self.w(f'double* const urow{ti} = sU + {ti * C * LD}u + ei * {N * LD}u + l;')
        if t.R is None:
          for j in range(N):
            self.w(f'urow{ti}[{j * LD}] = q{j};')
          continue
        if t.R.kind == 'batched':
          nrp = _pad(t.R.storage_size(), 2)
          if L['prefetch']:
            self.w(f'const double* const rq{ti} = sS + {L["stage_off"][t.R.name]}u + ei * {nrp}u;')
          else:
            self.w(f'const double* const rq{ti} = sR + {L["r_off"][t.R.name]}u + ei * {nrp}u;')
          rv = lambda pos, ti=ti: f'rq{ti}[{pos}]'
        else:
          rv = lambda pos, t=t: f'__ldg({t.R.name} + {pos})'
        look = t.R.sparse_lookup() if t.R.sparse else None
        for j in range(N):
          expr = '0.0'
          for m in range(P):
            pos = look.get((m, j)) if look is not None else j * P + m
            if pos is not None:
              expr = f'fma(q{m}, {rv(pos)}, {expr})'
          self.w(f'urow{ti}[{j * LD}] = {expr};')
      self.close()

  def _mma_phase(self):
    s, L = self.s, self.L
    MB, NS, NB, LD, C, MP = self.MB, self.NS, self.NB, L['LD'], L['C'], L['MP']
    nbw = -(-NB // NS)
    self.w(f'double acc[{nbw}][2];')
    self.w('#pragma unroll')
    self.w(f'for (int i = 0; i < {nbw}; ++i) {{ acc[i][0] = 0.0; acc[i][1] = 0.0; }}')
    self.w(f'const double* const ap = sA + (8u * mb + fr) * {LD}u + fq;')
    self.w(f'const double* const up = sU + (8u * ns + fr) * {LD}u + fq;')
    full = NB % NS == 0
    if not full:
      self.w(f'const bool last_ok = ns + {NS * (nbw - 1)}u < {NB}u;')
    for ti, t in enumerate(s.terms):
      ksteps = _pad(t.K, 4) // 4
      self.w('#pragma unroll')
      self.open(f'for (int kk = 0; kk < {ksteps}; ++kk)')
      self.w(f'const double a = ap[{ti * MP * LD} + 4 * kk];')
      for i in range(nbw):
        stmt = (f'tfb_dmma::mma(acc[{i}][0], acc[{i}][1], a, up[{ti * C * LD + i * 8 * NS * LD} + 4 * kk]);')
        if i == nbw - 1 and not full:
          stmt = f'if (last_ok) {stmt}'
        self.w(stmt)
      self.close()

  def _epilogue(self):
    s, L, BT, TE = self.s, self.L, self.BT, self.TE
    M, N, LDO, NS = s.M, s.N, L['LDO'], self.NS
    nbw = -(-self.NB // NS)
    full = self.NB % NS == 0
    self.w('__syncthreads();  // U is dead: the region becomes the output stage')
    guard = '' if M % 8 == 0 else f'if (8u * mb + fr < {M}u) '
    self.open(guard + '')
    for i in range(nbw):
      cond = 'last_ok' if (i == nbw - 1 and not full) else None
      base = f'(8u * (ns + {NS * i}u) + 2u * fq) * {LDO}u + 8u * mb + fr'
      st = f'sU[{base}] = acc[{i}][0]; sU[{base} + {LDO}u] = acc[{i}][1];'
      self.w(f'if ({cond}) {{ {st} }}' if cond else st)
    self.close()
    self.w('__syncthreads();')
    o = s.out
    vol = M * N
    self.open(f'for (unsigned q = threadIdx.x; q < {TE * vol}u; q += {BT}u)')
    self.w(f'const unsigned ei = q / {vol}u, r = q - ei * {vol}u, j = r / {M}u, m = r - j * {M}u;')
    self.w('const size_t e = e0 + ei;')
    self.open('if (e < numElements && (flags == nullptr || flags[e] != 0u))')
    self.w(f'double* const dst = {self._elem_ptr(o, "e")} + r;')
    val = f'sU[(ei * {N}u + j) * {LDO}u + m]'
    self.w(f'*dst {"+=" if s.accumulate else "="} {val};')
    self.close()
    self.close()
    self.w('__syncthreads();')

  # ------------------------------------------------------------------ kernel + launch
  def emit(self, globals_):
    s, L, BT, TE, b = self.s, self.L, self.BT, self.TE, self.base
    kname = f'kernel_{b}'
    self.w(DMMA_HELPERS)
    if self.L['prefetch']:
      from .colprog import CP_HELPERS
      self.w(CP_HELPERS)
    self.w(f'// generated by tensorforge_b200 (strategy: dmma, tile={TE} elements, C={L["C"]} columns, '
           f'{self.MB}x{self.NS} warps, LD={L["LD"]}, LDO={L["LDO"]})')
    self.w('// meta data:')
    for o in self.chain.operands:
      self.w(f'// {o.tensor.gen_descr()}')
    for st in self.chain.stages:
      self.w(f'// {st.descr}')
    self._a_tables()
    self.w(f'__global__ void __launch_bounds__({BT}, 1) {kname}({", ".join(self.params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(16) unsigned char tfb_smem_raw[];')
    self.w('double* const smem = reinterpret_cast<double*>(tfb_smem_raw);')
    self.w('double* const sA = smem;')
    self.w(f'double* const sU = smem + {L["A"]};')
    self.w(f'double* const sR = smem + {L["A"] + L["region"]};')
    if L['prefetch']:
      self.w(f'double* const sS = smem + {L["A"] + L["region"] + L["R"]};')
    self.w(f'const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;')
    self.w(f'const unsigned mb = warp % {self.MB}u, ns = warp / {self.MB}u;')
    self.w('const unsigned fr = lane >> 2, fq = lane & 3u;')
    self._stage_a()
    self.w(f'const size_t numTiles = (numElements + {TE - 1}u) / {TE}u;')
    pf = L['prefetch']
    if pf:
      self.open('if (blockIdx.x < numTiles)')
      self._prefetch('(size_t)blockIdx.x')
      self.close()
      self.w('tfb_cp::commit();')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x)')
    self.w(f'const size_t e0 = tile * {TE}u;')
    if pf:
      self.w('tfb_cp::wait_all();')
      self.w('__syncthreads();')
    elif L['r_off']:
      self._stage_r()
      self.w('__syncthreads();')
    self._u_phase()
    self.w('__syncthreads();')
    if pf:
      self.w('// the stage is consumed: fetch the next tile while the MMAs run')
      self.open('if (tile + gridDim.x < numTiles)')
      self._prefetch('tile + gridDim.x')
      self.close()
      self.w('tfb_cp::commit();')
    self._mma_phase()
    self._epilogue()
    self.close()
    if pf:
      self.w('tfb_cp::wait_all();')
    self.ind -= 1
    self.w('}')
    return '\n'.join(self.lines), self._launch(globals_, kname), ''

  def _launch(self, globals_, kname):
    args = []
    for t, _ in globals_:
      args.append(t.name)
      if t.addressing.name not in ('NONE', 'SCALAR'):
        args.append(f'{t.name}_extraOffset')
    args += ['numElements', 'flags']
    smem = self.L['total'] * 8
    pre = [f'  static int occ[64];',
           f'  if (device < 64 && occ[device] == 0) {{',
           f'    int sms = 0, per = 0;',
           f'    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);',
           f'    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, {kname}, {self.BT}, {smem});',
           f'    occ[device] = (per > 0 ? per : 1) * (sms > 0 ? sms : 1);',
           f'  }}',
           f'  const size_t cap = device < 64 ? (size_t)occ[device] : (size_t)1024;',
           f'  if (grid.x > cap) grid.x = (unsigned)cap;']
    self.plan.smem_bytes = smem
    return {'kernel': kname, 'block': self.BT, 'elements_per_block': self.TE, 'smem': smem, 'args': args,
            'grid': f'(numElements + {self.TE - 1}u) / {self.TE}u', 'pre': '\n'.join(pre)}
