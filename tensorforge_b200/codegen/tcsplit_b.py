"""tcgen05 TF32x3 generator, operand form B: the per-element input is the MMA's B operand.

For shared-left chains whose terms all read the same per-element input B_e,

    out_e = sum_t A_t * B_e * R_{e,t}      (A_t shared M x K, B_e K x P, R_{e,t} P x N)

this form computes W_t = A_t * B_e on the tensor cores and applies R_{e,t} in the epilogue:

  * MMA: M = 128 TMEM lanes = two terms' A stacked ([A_0; A_1], each padded to 64 rows;
    an odd last term is stacked with itself), N = TE * P flat input columns (e, m) of a
    tile of TE elements (padded to 16, at most 64), K = K padded to the 8-value step. Both
    operands come from shared memory in the canonical no-swizzle K-major layout: A split
    once per CTA into hi + lo, B_e split per tile by the producers straight from the staged
    column-major input (a column of B_e is already K-contiguous), so no per-element
    product is formed on CUDA cores before the MMA.
  * Precision: hi = value rounded to nearest TF32, lo = the remainder (the tensor core
    reads its TF32 part); the three products hi*hi, hi*lo and lo*hi accumulate in one TMEM
    accumulator (plan option acc=1) or hi*hi apart from the cross terms (acc=2), summed in
    FP32 in the epilogue.
  * Epilogue: lane i of a stacked block holds row i of W_t for every flat column; each
    producer reads its row of one element's P columns (tcgen05.ld), sums the two
    accumulators and applies R_{e,t} with its compile-time pattern unrolled. The two
    lane halves (terms 0 / 1) combine through the shared staging buffer, which is written
    back with one bulk store (cp.async.bulk, shared -> global) when the output is strided,
    aligned and unmasked, else element by element.
  * Pipelining: two accumulator sets (TMEM columns 2 x blocks x accumulators x N <= 512)
    and one or two B tiles (plan option bbuf), so the tensor cores work on tile n while the
    producers run the epilogue of tile n-1 (and, with two B tiles, split tile n+1). The
    tile is the largest element count that fits TMEM and shared memory. Every mbarrier
    wait is bounded (error word `tfb_kernel_error_<name>`), named barriers are taken
    uniformly by all producers.
"""
from .tcsplit import HELPERS, _pad, H_GROUPS

TCB_HELPERS = r'''
#ifndef TFB_TCB_HELPERS
#define TFB_TCB_HELPERS
namespace tfb_tcb {
// D (tmem) (+)= A (smem descriptor) * B (smem descriptor), kind::tf32
__device__ __forceinline__ void mma_ss_tf32(unsigned d_tmem, uint64_t a_desc, uint64_t b_desc, unsigned idesc, unsigned accum) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}"
               :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accum) : "memory");
}
__device__ __forceinline__ void ld_x1(unsigned taddr, unsigned* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(v[0]) : "r"(taddr) : "memory");
}
__device__ __forceinline__ void ld_x2(unsigned taddr, unsigned* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];" : "=r"(v[0]), "=r"(v[1]) : "r"(taddr) : "memory");
}
__device__ __forceinline__ void ld_x4(unsigned taddr, unsigned* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "r"(taddr) : "memory");
}
}  // namespace tfb_tcb
#endif
'''

MAX_ROWS = 64      # rows of one stacked term (half of the 128 lanes)
SMEM_MAX = 227 * 1024


def blocks_of(nterms):
  """Stacked A blocks: (term in lanes 0-63, term in lanes 64-127, split). A split block holds
  one term twice and its elements are divided between the two lane halves."""
  if nterms == 1:
    return [(0, 0, True)]
  if nterms == 2:
    return [(0, 1, False)]
  if nterms == 3:
    return [(0, 1, False), (2, 2, True)]
  if nterms == 4:
    return [(0, 1, False), (2, 3, False)]
  return None


def _sizes(shape, te, acc, bbuf, nrb=2):
  terms = shape.terms
  B = terms[0].B
  K, P, M, N = terms[0].K, terms[0].P, shape.M, shape.N
  n_mma = _pad(te * P, 16)
  kpad = _pad(K, 8)
  blocks = blocks_of(len(terms))
  a_bytes = 128 * kpad * 4
  b_bytes = n_mma * kpad * 4
  vol_b = _pad(B.element_volume(), 4)
  r_off, r_vals = {}, 0
  for ti, t in enumerate(terms):
    if t.R is not None:
      r_off[ti] = r_vals
      r_vals += te * _pad(t.R.storage_size(), 4)
  vol_o = M * N
  off = 0
  off_a = off
  off += len(blocks) * 2 * a_bytes
  off_b = off
  off += bbuf * 2 * b_bytes
  off_raw = off
  off += _pad(te * vol_b * 4, 128)
  off_r = off
  off += _pad(nrb * r_vals * 4, 128)
  off_out = off
  off += _pad(te * vol_o * 4, 128)
  off_bar = off
  total = off + 256
  tmem = 2 * len(blocks) * acc * n_mma
  return dict(te=te, n_mma=n_mma, kpad=kpad, K=K, P=P, M=M, N=N, blocks=blocks, a_bytes=a_bytes,
              b_bytes=b_bytes, vol_b=vol_b, r_off=r_off, r_vals=r_vals, vol_o=vol_o, off_a=off_a, off_b=off_b,
              off_raw=off_raw, off_r=off_r, off_out=off_out, off_bar=off_bar, total=total,
              hsplit=(te + 1) // 2, acc=acc, bbuf=bbuf, tmem=tmem, nrb=nrb)


def layout_b(shape, acc=1, bbuf=1, te=None, ws=0):
  """Sizes and shared-memory offsets of form B, or None when the chain does not fit it.

  acc: accumulators per block (1: all three split products in one; 2: hi*hi apart from the
  cross terms); bbuf: B tiles in shared memory (2 lets the producers split tile n+1 while the
  tensor cores still read tile n). The tile is the largest number of whole elements whose
  flat columns (padded to 16, at most 256) fit two accumulator sets in the 512 TMEM columns
  and whose buffers fit in shared memory."""
  terms = shape.terms
  if len(terms) < 1 or len(terms) > 4 or shape.accumulate or shape.epilogue:
    return None
  B = terms[0].B
  if any(t.B is not B for t in terms) or B.kind != 'batched' or B.sparse:
    return None
  if B.addressing.name not in ('STRIDED', 'PTR_BASED'):
    return None
  K, P, M, N = terms[0].K, terms[0].P, shape.M, shape.N
  if M > MAX_ROWS or K % 4 != 0 or B.element_volume() != K * P:
    return None
  for t in terms:
    if t.R is None:
      if P != N:
        return None
    elif t.R.kind != 'batched' or t.R.shape[0] != P or t.R.shape[1] != N:
      return None
  out = shape.out
  if out.addressing.name not in ('STRIDED', 'PTR_BASED') or out.sparse:
    return None
  cands = [te] if te is not None else range(256 // P, 0, -1)
  for t_e in cands:
    if t_e < 1 or _pad(t_e * P, 16) > 256:
      continue
    L = _sizes(shape, t_e, acc, bbuf, 3 if ws else 2)
    if L['tmem'] <= 512 and L['total'] <= SMEM_MAX:
      return L
  return None


class _TCB:
  WAIT_LIMIT = 1 << 26

  def __init__(self, chain, shape, plan_, ctx, base):
    self.chain = chain
    self.s = shape
    self.plan = plan_
    self.ctx = ctx
    self.base = base
    p = plan_.params
    self.ws = int(p.get('ws', 0))
    self.L = layout_b(shape, p.get('acc', 1), p.get('bbuf', 1), p.get('te'), self.ws)
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
    params = []
    for t, _ in globals_:
      dt = 'float' if t.datatype is None else str(t.datatype)
      if t.addressing.name == 'SCALAR':
        params.append(f'{dt} {t.name}')
      else:
        const = 'const ' if t.direction.name == 'SOURCE' else ''
        params.append(f'{const}{dt}{t.addressing.to_pointer()} __restrict__ {t.name}')
        if t.addressing.name != 'NONE':
          params.append(f'unsigned {t.name}_extraOffset')
    params += ['size_t numElements', 'const unsigned* __restrict__ flags']
    return params

  def _elem_ptr(self, op, e):
    a = op.addressing.name
    if a == 'STRIDED':
      return f'({op.name} + ({e}) * {op.element_volume()}u + {op.name}_extraOffset)'
    if a == 'PTR_BASED':
      return f'({op.name}[{e}] + {op.name}_extraOffset)'
    return f'{op.name}'

  def _copy(self, op, vals, dst, tile_expr, NP, tid='ptid'):
    """cp.async `vals` values per element of tile `tile_expr` to `dst` + ei * pad4(vals).

    Pointer-array operands are copied one element per warp at a time, so the element's
    pointer is loaded once per warp instead of once per 16-byte chunk."""
    te = self.L['te']
    vp = _pad(vals, 4)
    self.open('')
    self.w(f'const size_t ce0 = ({tile_expr}) * {te}u;')
    if op.addressing.name == 'PTR_BASED':
      nw = NP // 32
      self.open(f'for (unsigned ei = ({tid}) >> 5; ei < {te}u; ei += {nw}u)')
      self.w('const size_t ee = ce0 + ei;')
      self.w('if (ee >= numElements) break;')
      self.w(f'const float* const sbase = {self._elem_ptr(op, "ee")};')
      self.w(f'float* const dbase = {dst} + ei * {vp}u;')
      if vals % 4 == 0:
        self.w('const bool al = (reinterpret_cast<uintptr_t>(sbase) & 15u) == 0u;')
        self.open(f'for (unsigned c4 = ({tid}) & 31u; c4 < {vals // 4}u; c4 += 32u)')
        self.w('const float* src = sbase + 4u * c4;')
        self.w('float* dst = dbase + 4u * c4;')
        self.w('if (al) tfb_tc::cp_async16(dst, src);')
        self.w('else { tfb_tc::cp_async4(dst, src); tfb_tc::cp_async4(dst + 1, src + 1); '
               'tfb_tc::cp_async4(dst + 2, src + 2); tfb_tc::cp_async4(dst + 3, src + 3); }')
        self.close()
      else:
        self.w(f'for (unsigned c = ({tid}) & 31u; c < {vals}u; c += 32u) tfb_tc::cp_async4(dbase + c, sbase + c);')
      self.close()
      self.close()
      return
    if vals % 4 == 0:
      self.open(f'for (unsigned q = ptid; q < {te * vals // 4}u; q += {NP}u)')
      self.w(f'const unsigned ei = q / {vals // 4}u, c4 = q - ei * {vals // 4}u;')
      self.w('const size_t ee = ce0 + ei;')
      self.open('if (ee < numElements)')
      self.w(f'const float* src = {self._elem_ptr(op, "ee")} + 4u * c4;')
      self.w(f'float* dst = {dst} + ei * {vp}u + 4u * c4;')
      self.w('if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0u) tfb_tc::cp_async16(dst, src);')
      self.w('else { tfb_tc::cp_async4(dst, src); tfb_tc::cp_async4(dst + 1, src + 1); '
             'tfb_tc::cp_async4(dst + 2, src + 2); tfb_tc::cp_async4(dst + 3, src + 3); }')
      self.close()
      self.close()
    else:
      self.open(f'for (unsigned q = ptid; q < {te * vals}u; q += {NP}u)')
      self.w(f'const unsigned ei = q / {vals}u, c = q - ei * {vals}u;')
      self.w('const size_t ee = ce0 + ei;')
      self.w(f'if (ee < numElements) tfb_tc::cp_async4({dst} + ei * {vp}u + c, {self._elem_ptr(op, "ee")} + c);')
      self.close()
    self.close()

  def _store_elements(self, out, vol_o, tid, nthreads):
    """Staged tile -> the output, one element per warp (its pointer and flag read once),
    skipping masked elements."""
    nw = nthreads // 32
    self.open(f'for (unsigned ei = ({tid}) >> 5; ei < nvalid; ei += {nw}u)')
    self.w('const size_t ee = pe0 + ei;')
    self.w('if (flags != nullptr && flags[ee] == 0u) continue;')
    self.w(f'float* const obase_e = {self._elem_ptr(out, "ee")};')
    self.w(f'for (unsigned c = ({tid}) & 31u; c < {vol_o}u; c += 32u) obase_e[c] = stg[ei * {vol_o}u + c];')
    self.close()

  def _load_b(self, tile_expr, NP):
    B = self.s.terms[0].B
    self._copy(B, B.element_volume(), 'raw', tile_expr, NP)

  def _load_r(self, tile_expr, rbuf, NP):
    L = self.L
    for ti, off in L['r_off'].items():
      R = self.s.terms[ti].R
      self._copy(R, R.storage_size(), f'({rbuf} + {off})', tile_expr, NP)

  def _col(self, buf, blk, acc):
    L = self.L
    nb, na = len(L['blocks']), L['acc']
    return f'({buf}) * {nb * na * L["n_mma"]}u + {(blk * na + acc) * L["n_mma"]}u'

  def emit(self, globals_):
    s, L, b = self.s, self.L, self.base
    kname = f'kernel_{b}'
    H = H_GROUPS
    NP = 128 * H
    nthreads = NP + 32
    te, n_mma, kpad, K, P, M, N = L['te'], L['n_mma'], L['kpad'], L['K'], L['P'], L['M'], L['N']
    blocks = L['blocks']
    nb = len(blocks)
    sbo_a = (kpad // 4) * 128
    sbo_b = (kpad // 4) * 128
    ksteps = kpad // 8
    lim = self.WAIT_LIMIT
    idesc = (1 << 4) | (2 << 7) | (2 << 10) | ((n_mma >> 3) << 17) | ((128 >> 4) << 24)
    BAR_STAGE, BAR_BFULL, BAR_BFREE, BAR_DFULL, BAR_DFREE = 0, 1, 3, 5, 7
    BAR_RFULL, BAR_RFREE = 9, 9 + L['nrb']
    nbars = 9 + 2 * L['nrb'] if self.ws else 9
    out = s.out
    smem = max(L['total'], 120 * 1024)
    self.plan.smem_bytes = smem

    # gather tables: row r of block `blk` (lanes 0-63: term lo, 64-127: term hi), column k
    gathers = []
    for blk, (tlo, thi, _) in enumerate(blocks):
      tbl = []
      for r in range(128):
        t = s.terms[tlo if r < 64 else thi]
        i = r & 63
        look = t.A.sparse_lookup() if t.A.sparse else None
        for k in range(kpad):
          if i < M and k < K:
            tbl.append(k * t.A.shape[0] + i if look is None else look.get((i, k), -1))
          else:
            tbl.append(-1)
      gathers.append(tbl)

    self.w(HELPERS)
    self.w(TCB_HELPERS)
    self.w(f'// generated by tensorforge_b200 (strategy: tcsplit form B, tf32x3, tile={te} elements, '
           f'N={n_mma}, K={kpad}, {nb} stacked block(s), smem={L["total"]} B)')
    self.w('// meta data:')
    for o in self.chain.operands:
      self.w(f'// {o.tensor.gen_descr()}')
    for st in self.chain.stages:
      self.w(f'// {st.descr}')
    for blk, tbl in enumerate(gathers):
      self.w(f'__device__ const short agather{blk}_{b}[{len(tbl)}] = {{{", ".join(str(x) for x in tbl)}}};')
    self.w(f'__device__ unsigned tfb_err_{b} = 0u;')
    self.w(f'extern "C" int tfb_kernel_error_{b}(void* stream) {{')
    self.w('  unsigned v = 0, z = 0;')
    self.w('  cudaStream_t st = static_cast<cudaStream_t>(stream);')
    self.w(f'  cudaMemcpyFromSymbolAsync(&v, tfb_err_{b}, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);')
    self.w(f'  cudaMemcpyToSymbolAsync(tfb_err_{b}, &z, sizeof(unsigned), 0, cudaMemcpyHostToDevice, st);')
    self.w('  cudaStreamSynchronize(st);')
    self.w('  return (int)v;')
    self.w('}')
    self.w(f'__global__ void __launch_bounds__({nthreads}, 1) {kname}({", ".join(self.params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(1024) unsigned char tfb_smem_raw[];')
    self.w(f'uint64_t* const bars = reinterpret_cast<uint64_t*>(tfb_smem_raw + {L["off_bar"]});')
    self.w(f'unsigned* const tmem_slot = reinterpret_cast<unsigned*>(bars + {nbars});')
    self.w(f'float* const raw = reinterpret_cast<float*>(tfb_smem_raw + {L["off_raw"]});')
    self.w(f'float* const rbase = reinterpret_cast<float*>(tfb_smem_raw + {L["off_r"]});')
    self.w(f'float* const stg = reinterpret_cast<float*>(tfb_smem_raw + {L["off_out"]});')
    self.w('const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;')
    self.w(f'const size_t numTiles = (numElements + {te - 1}u) / {te}u;')
    # ---- setup: stacked A blocks (hi / lo), barriers, TMEM
    for blk in range(nb):
      hi_off = L['off_a'] + blk * 2 * L['a_bytes']
      lo_off = hi_off + L['a_bytes']
      tlo, thi, _ = blocks[blk]
      self.open(f'for (int q = threadIdx.x; q < {128 * kpad}; q += blockDim.x)')
      self.w(f'const int r = q / {kpad}, k = q - r * {kpad};')
      self.w(f'const int src = agather{blk}_{b}[q];')
      if tlo == thi:
        self.w(f'const float v = src >= 0 ? {s.terms[tlo].A.name}[src] : 0.0f;')
      else:
        self.w(f'const float v = src < 0 ? 0.0f : (r < 64 ? {s.terms[tlo].A.name}[src] : {s.terms[thi].A.name}[src]);')
      self.w(f'const unsigned boff = (r >> 3) * {sbo_a}u + (k >> 2) * 128u + (r & 7) * 16u + (k & 3) * 4u;')
      self.w('unsigned hb, lb;')
      self.w('tfb_tc::tf32_split(v, hb, lb);')
      self.w(f'*reinterpret_cast<unsigned*>(tfb_smem_raw + {hi_off} + boff) = hb;')
      self.w(f'*reinterpret_cast<unsigned*>(tfb_smem_raw + {lo_off} + boff) = lb;')
      self.close()
    # warp-specialized producers: warps 0-3 load and split (NS threads), warps 4-15 run the
    # epilogue (NE threads); otherwise all NP producers do both
    NS, NE = (128, NP - 128) if self.ws else (NP, NP)
    self.open('if (threadIdx.x == 0)')
    self.w(f'tfb_tc::mbar_init(&bars[{BAR_STAGE}], {NS}u);')
    for x in range(2):
      self.w(f'tfb_tc::mbar_init(&bars[{BAR_BFULL + x}], {NS}u);')
      self.w(f'tfb_tc::mbar_init(&bars[{BAR_BFREE + x}], 1u);')
      self.w(f'tfb_tc::mbar_init(&bars[{BAR_DFULL + x}], 1u);')
      self.w(f'tfb_tc::mbar_init(&bars[{BAR_DFREE + x}], {NE}u);')
    if self.ws:
      for x in range(L['nrb']):
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_RFULL + x}], {NS}u);')
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_RFREE + x}], {NE}u);')
    self.w('asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");')
    self.close()
    self.open('if (warp == 0)')
    self.w('tfb_tc::tmem_alloc(tmem_slot, 512u);')
    self.close()
    self.w('tfb_tc::fence_proxy_async();')
    self.w('tfb_tc::fence_before();')
    self.w('__syncthreads();')
    self.w('tfb_tc::fence_after();')
    self.w('const unsigned tmem = *tmem_slot;')
    self.w('bool ok = true;')
    # ---- MMA issuer
    self.open(f'if (warp == {4 * H})')
    self.open('if (lane == 0)')
    self.w('unsigned it = 0;')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles && ok; tile += gridDim.x, ++it)')
    bsel, bfull_par, _, _ = self._bbuf_exprs()
    self.w('const unsigned sb = it & 1u;             // accumulator set')
    self.w(f'const unsigned bs = {bsel};             // B tile buffer')
    self.w(f'if (!tfb_tc::mbar_wait(&bars[{BAR_BFULL} + bs], {bfull_par}, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 50u); break; }}')
    self.w(f'if (it >= 2u && !tfb_tc::mbar_wait(&bars[{BAR_DFREE} + sb], ((it - 2u) >> 1) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 51u); break; }}')
    self.w('tfb_tc::fence_after();')
    self.w(f'const unsigned bhi = tfb_tc::smem_u32(tfb_smem_raw + {L["off_b"]}) + bs * {2 * L["b_bytes"]}u;')
    self.w(f'const unsigned blo = bhi + {L["b_bytes"]}u;')
    for blk in range(nb):
      hi_off = L['off_a'] + blk * 2 * L['a_bytes']
      self.open('')
      self.w(f'const unsigned ahi = tfb_tc::smem_u32(tfb_smem_raw + {hi_off});')
      self.w(f'const unsigned alo = ahi + {L["a_bytes"]}u;')
      if L['acc'] == 2:
        self.w(f'const unsigned dm = tmem + {self._col("sb", blk, 0)}, dc = tmem + {self._col("sb", blk, 1)};')
      else:  # one accumulator takes all three split products
        self.w(f'const unsigned dm = tmem + {self._col("sb", blk, 0)}, dc = dm;')
      self.open(f'for (int ks = 0; ks < {ksteps}; ++ks)')
      self.w(f'const uint64_t ah = tfb_tc::smem_desc(ahi + ks * 256u, 128u, {sbo_a}u);')
      self.w(f'const uint64_t al = tfb_tc::smem_desc(alo + ks * 256u, 128u, {sbo_a}u);')
      self.w(f'const uint64_t bh = tfb_tc::smem_desc(bhi + ks * 256u, 128u, {sbo_b}u);')
      self.w(f'const uint64_t bl = tfb_tc::smem_desc(blo + ks * 256u, 128u, {sbo_b}u);')
      self.w(f'tfb_tcb::mma_ss_tf32(dm, ah, bh, {idesc}u, ks > 0 ? 1u : 0u);')
      self.w(f'tfb_tcb::mma_ss_tf32(dc, ah, bl, {idesc}u, {"ks > 0 ? 1u : 0u" if L["acc"] == 2 else "1u"});')
      self.w(f'tfb_tcb::mma_ss_tf32(dc, al, bh, {idesc}u, 1u);')
      self.close()
      self.close()
    self.w(f'tfb_tc::mma_commit(&bars[{BAR_BFREE} + bs]);')
    self.w(f'tfb_tc::mma_commit(&bars[{BAR_DFULL} + sb]);')
    self.close()
    self.close()
    self.close()
    # ---- producers
    if self.ws:
      self._split_team(lim, BAR_STAGE, BAR_BFULL, BAR_BFREE, BAR_RFULL, BAR_RFREE)
      self._epilogue_team(lim, BAR_DFULL, BAR_DFREE, BAR_RFULL, BAR_RFREE)
    else:
      self._producers(NP, lim, BAR_STAGE, BAR_BFULL, BAR_BFREE, BAR_DFULL, BAR_DFREE)
    # ---- teardown
    self.w('tfb_tc::fence_before();')
    self.w('__syncthreads();')
    self.open('if (warp == 0)')
    self.w('tfb_tc::fence_after();')
    self.w('tfb_tc::tmem_dealloc(tmem, 512u);')
    self.close()
    self.ind -= 1
    self.w('}')
    kernel = '\n'.join(self.lines)
    args = []
    for t, _ in globals_:
      args.append(t.name)
      if t.addressing.name not in ('NONE', 'SCALAR'):
        args.append(f'{t.name}_extraOffset')
    args += ['numElements', 'flags']
    pre = ('  int sms = 0;\n'
           '  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);\n'
           '  if (sms > 0 && grid.x > (unsigned)sms) grid.x = (unsigned)sms;')
    launch = {'kernel': kname, 'block': nthreads, 'elements_per_block': te, 'smem': smem, 'args': args,
              'grid': f'(numElements + {te - 1}u) / {te}u', 'pre': pre}
    return kernel, launch, ''

  # ------------------------------------------------------------------ producers
  def _producers(self, NP, lim, BAR_STAGE, BAR_BFULL, BAR_BFREE, BAR_DFULL, BAR_DFREE):
    s, L, b = self.s, self.L, self.base
    te, n_mma, kpad, K, P, M, N = L['te'], L['n_mma'], L['kpad'], L['K'], L['P'], L['M'], L['N']
    H = H_GROUPS
    self.open(f'else if (warp < {4 * H})')
    self.w('const unsigned ptid = threadIdx.x;')
    self.w('const unsigned quad = warp & 3u, grp = warp >> 2;')
    self.w('const unsigned tl = quad * 32u + lane;          // TMEM lane of this thread')
    self.w('const unsigned half = tl >> 6, row = tl & 63u;')
    self.w('const unsigned lane_addr = tmem + ((quad * 32u) << 16);')
    self.w('unsigned it = 0;')
    self.w('size_t prev_tile = 0; bool have_prev = false, pending = false;')
    self.open('if (blockIdx.x < numTiles)')
    self._load_b('(size_t)blockIdx.x', NP)
    self._load_r('(size_t)blockIdx.x', 'rbase', NP)
    self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
    self.w('pending = true;')
    self.close()
    self.open('for (size_t tile = blockIdx.x; ; tile += gridDim.x, ++it)')
    self.w('// uniform control flow around named barriers: a timeout anywhere stops every')
    self.w('// producer at the next tile boundary (barrier-wide OR), never mid-tile')
    self.w(f'if (tfb_tc::any_sync(1, {NP}, !ok)) break;')
    self.w('const bool more = tile < numTiles;')
    self.w('const size_t ntile = tile + gridDim.x;')
    self.w('const bool has_next = more && ntile < numTiles;')
    self.open('if (more)')
    self.w(f'if (!tfb_tc::mbar_wait(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 60u); }}')
    self.w('pending = false;')
    bsel, _, free_cond, free_par = self._bbuf_exprs()
    self.w(f'if ({free_cond} && !tfb_tc::mbar_wait(&bars[{BAR_BFREE} + {bsel}], {free_par}, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 61u); }}')
    self._split(NP, bsel)
    self.w('tfb_tc::fence_proxy_async();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{BAR_BFULL} + {bsel}]);')
    self.close()
    self.w(f'tfb_tc::named_sync(1, {NP});   // the raw stage has been read')
    self.open('if (has_next)')
    self._load_b('ntile', NP)
    self.close()
    self.open('if (have_prev)')
    self._epilogue(NP, lim, BAR_DFULL, BAR_DFREE)
    self.close()
    self.open('if (has_next)')
    self._load_r('ntile', f'(rbase + ((it + 1u) & 1u) * {L["r_vals"]}u)', NP)
    self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
    self.w('pending = true;')
    self.close()
    self.w('if (!more) break;')
    self.w('prev_tile = tile; have_prev = true;')
    self.close()
    self.w('// a stage load still in flight after an abort must land before the CTA exits')
    self.w(f'if (pending && !tfb_tc::mbar_wait(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) atomicMax(&tfb_err_{b}, 62u);')
    self.w('tfb_tc::cp_async_wait_all();')
    self.w('if (ptid == 0) tfb_tc::bulk_wait();')
    self.close()

  def _bbuf_exprs(self):
    """(buffer of tile `it`, BFULL parity, BFREE wait condition, BFREE parity)."""
    if self.L['bbuf'] == 1:
      return '0u', 'it & 1u', 'it >= 1u', '(it - 1u) & 1u'
    return '(it & 1u)', '(it >> 1) & 1u', 'it >= 2u', '((it - 2u) >> 1) & 1u'

  def _split(self, NP, bsel, tid='ptid'):
    """raw stage (column-major K x P per element) -> B tile hi / lo in canonical K-major layout;
    row n = flat column (e, m), K contiguous (a column of B_e), 4 values per item. Consecutive
    threads take consecutive rows n, so each 8-row core matrix is one conflict-free 128-byte
    store; lo = value - hi is passed unrounded (the tensor core reads its TF32 part)."""
    L = self.L
    te, kpad, K, P = L['te'], L['kpad'], L['K'], L['P']
    k4 = kpad // 4
    nr = te * P
    sbo = (kpad // 4) * 128
    self.open('')
    self.w(f'unsigned char* const bh = tfb_smem_raw + {L["off_b"]} + {bsel} * {2 * L["b_bytes"]}u;')
    self.w(f'unsigned char* const bl = bh + {L["b_bytes"]}u;')
    self.open(f'for (unsigned q = {tid}; q < {nr * k4}u; q += {NP}u)')
    self.w(f'const unsigned l4 = q / {nr}u, n = q - l4 * {nr}u;')
    self.w(f'const unsigned ei = n / {P}u, m = n - ei * {P}u;')
    self.w('float4 x = make_float4(0.0f, 0.0f, 0.0f, 0.0f);')
    self.w(f'if (l4 < {K // 4}u) x = *reinterpret_cast<const float4*>(raw + ei * {L["vol_b"]}u + m * {K}u + 4u * l4);')
    self.w('uint4 h, l;')
    self.w('h.x = tfb_tc::tf32_rna(x.x); l.x = __float_as_uint(x.x - __uint_as_float(h.x));')
    self.w('h.y = tfb_tc::tf32_rna(x.y); l.y = __float_as_uint(x.y - __uint_as_float(h.y));')
    self.w('h.z = tfb_tc::tf32_rna(x.z); l.z = __float_as_uint(x.z - __uint_as_float(h.z));')
    self.w('h.w = tfb_tc::tf32_rna(x.w); l.w = __float_as_uint(x.w - __uint_as_float(h.w));')
    self.w(f'const unsigned off = (n >> 3) * {sbo}u + l4 * 128u + (n & 7u) * 16u;')
    self.w('*reinterpret_cast<uint4*>(bh + off) = h;')
    self.w('*reinterpret_cast<uint4*>(bl + off) = l;')
    self.close()
    self.close()

  def _ld_cols(self, base_expr, c0, name, count):
    """tcgen05.ld of columns [c0, c0 + count) past `base_expr` (a multiple of 64 columns)
    into unsigned name[count], in chunks of 1/2/4/8 columns each aligned to its width."""
    self.w(f'unsigned {name}[{count}];')
    c = 0
    while c < count:
      col = c0 + c
      width = 8
      while width > 1 and (col % width != 0 or c + width > count):
        width //= 2
      fn = {8: 'tfb_tc::ld_x8', 4: 'tfb_tcb::ld_x4', 2: 'tfb_tcb::ld_x2', 1: 'tfb_tcb::ld_x1'}[width]
      self.w(f'{fn}({base_expr} + {col}u, {name} + {c});')
      c += width

  def _term_partial(self, ti, e, blk, acc_name):
    """acc_name[j] += sum_m W_ti[row, (e, m)] R_ti[m, j] for this thread's row; e is a
    compile-time element index within the tile."""
    s, L = self.s, self.L
    P, N = L['P'], L['N']
    t = s.terms[ti]
    nmma = L['n_mma']
    self.open('')
    na = L['acc']
    base = f'(lane_addr + pb * {len(L["blocks"]) * na * nmma}u)'
    self._ld_cols(base, blk * na * nmma + e * P, 'wm', P)
    if na == 2:
      self._ld_cols(base, blk * na * nmma + nmma + e * P, 'wc', P)
    self.w('tfb_tc::ld_wait();')
    for m in range(P):
      if na == 2:
        self.w(f'const float w{m} = __uint_as_float(wm[{m}]) + __uint_as_float(wc[{m}]);')
      else:
        self.w(f'const float w{m} = __uint_as_float(wm[{m}]);')
    if t.R is None:
      for j in range(N):
        self.w(f'{acc_name}[{j}] += w{j};')
    else:
      nr = t.R.storage_size()
      rp = _pad(nr, 4)
      self.w(f'const float4* const rq = reinterpret_cast<const float4*>(rprev + {L["r_off"][ti] + e * rp}u);')
      for v in range((nr + 3) // 4):
        self.w(f'const float4 r{v} = rq[{v}];')
      comp = ['x', 'y', 'z', 'w']
      look = t.R.sparse_lookup() if t.R.sparse else None
      for j in range(N):
        terms = []
        for m in range(P):
          pos = look.get((m, j)) if look is not None else j * P + m
          if pos is not None:
            terms.append((m, pos))
        if not terms:
          continue
        expr = f'{acc_name}[{j}]'
        for m, pos in terms:
          expr = f'fmaf(w{m}, r{pos // 4}.{comp[pos % 4]}, {expr})'
        self.w(f'{acc_name}[{j}] = {expr};')
    self.close()

  def _epilogue(self, NP, lim, BAR_DFULL, BAR_DFREE):
    s, L, b = self.s, self.L, self.base
    te, P, M, N = L['te'], L['P'], L['M'], L['N']
    H = H_GROUPS
    blocks = L['blocks']
    hs = L['hsplit']
    per = (te + H - 1) // H              # elements per producer group
    out = s.out
    vol_o = L['vol_o']
    self.w('const unsigned pb = (it - 1u) & 1u;')
    self.w(f'if (!tfb_tc::mbar_wait(&bars[{BAR_DFULL}] + pb, ((it - 1u) >> 1) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 63u); }}')
    self.w('tfb_tc::fence_after();')
    self.w(f'const float* const rprev = rbase + pb * {L["r_vals"]}u;')
    for k in range(per):
      self.w(f'float p{k}[{N}];')
      self.w('#pragma unroll')
      self.w(f'for (int j = 0; j < {N}; ++j) p{k}[j] = 0.0f;')
    # warp-uniform branches: grp (the group's elements) and half (the lane quadrant's term)
    # are the same across a warp; elements are compile-time inside each branch so the
    # tensor-memory column offsets are constants
    for g in range(H):
      self.open(f'{"if" if g == 0 else "else if"} (grp == {g}u)')
      for k in range(per):
        e = g + k * H
        if e >= te:
          continue
        for blk, (tlo, thi, split) in enumerate(blocks):
          if split:
            self.open(f'if (half == {0 if e < hs else 1}u)')
            self._term_partial(tlo, e, blk, f'p{k}')
            self.close()
          else:
            self.open('if (half == 0u)')
            self._term_partial(tlo, e, blk, f'p{k}')
            self.close()
            self.open('else')
            self._term_partial(thi, e, blk, f'p{k}')
            self.close()
      self.close()
    self.w('tfb_tc::fence_before();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{BAR_DFREE}] + pb);')
    # combine the two lane halves in the staging buffer (the previous bulk store has read it)
    self.w(f'const size_t pe0 = prev_tile * {te}u;')
    self.w(f'const unsigned nvalid = (unsigned)((numElements - pe0) < {te}u ? (numElements - pe0) : {te}u);')
    self.w('if (ptid == 0) tfb_tc::bulk_wait_read();')
    self.w(f'tfb_tc::named_sync(1, {NP});')
    first_half1_assigns = len(s.terms) == 1   # half 1 holds elements half 0 does not touch
    for phase in (0, 1):
      self.open(f'if (half == {phase}u && row < {M}u)')
      for k in range(per):
        e = f'(grp + {k * H}u)'
        self.open(f'if ({e} < nvalid)')
        self.w(f'float* const dst = stg + {e} * {vol_o}u + row;')
        if phase == 0:
          cond = '' if not blocks[0][2] else f'if ({e} < {hs}u) '
          self.w(f'{cond}{{ ' + ' '.join(f'dst[{j * M}] = p{k}[{j}];' for j in range(N)) + ' }')
        else:
          if first_half1_assigns:
            self.w(f'if ({e} >= {hs}u) {{ ' + ' '.join(f'dst[{j * M}] = p{k}[{j}];' for j in range(N)) + ' }')
          else:
            self.w('{ ' + ' '.join(f'dst[{j * M}] += p{k}[{j}];' for j in range(N)) + ' }')
        self.close()
      self.close()
      if phase == 1:
        self.w('tfb_tc::fence_proxy_async();   // staged values visible to the bulk store')
      self.w(f'tfb_tc::named_sync(1, {NP});')
    # write back
    bulk_ok = out.addressing.name == 'STRIDED' and out.element_volume() == vol_o and (vol_o * 4) % 16 == 0
    if bulk_ok:
      self.w(f'float* const obase = {out.name} + pe0 * {out.element_volume()}u + {out.name}_extraOffset;')
      self.w('const bool bulk = flags == nullptr && ((reinterpret_cast<uintptr_t>(obase) & 15u) == 0u);')
      self.open('if (bulk)')
      self.open('if (ptid == 0)')
      self.w(f'tfb_tc::bulk_store(obase, stg, nvalid * {vol_o * 4}u);')
      self.close()
      self.close()
      self.open('else')
    else:
      self.open('')
    self._store_elements(out, vol_o, 'ptid', NP)
    self.close()

  # ------------------------------------------------------------------ warp-specialized producers
  def _split_team(self, lim, BAR_STAGE, BAR_BFULL, BAR_BFREE, BAR_RFULL, BAR_RFREE):
    """Warps 0-3: per tile, wait for the staged input, split it into the free B buffer, then
    stage the next tile's input and R values (R in a ring of nrb buffers, each reloaded only
    after the epilogue team released it)."""
    L, b = self.L, self.base
    NS = 128
    nrb = L['nrb']
    has_r = bool(L['r_off'])
    self.open('if (warp < 4)')
    self.w('const unsigned ptid = threadIdx.x;')
    self.w('unsigned it = 0;')
    self.w('bool pending = false;')
    self.open('if (blockIdx.x < numTiles)')
    self._load_b('(size_t)blockIdx.x', NS)
    self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
    if has_r:
      self._load_r('(size_t)blockIdx.x', 'rbase', NS)
      self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_RFULL}]);')
    self.w('pending = true;')
    self.close()
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it)')
    self.w(f'if (tfb_tc::any_sync(2, {NS}, !ok)) break;')
    self.w('const size_t ntile = tile + gridDim.x;')
    self.w('const bool has_next = ntile < numTiles;')
    self.w(f'if (!tfb_tc::mbar_wait(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 70u); }}')
    self.w('pending = false;')
    bsel, _, free_cond, free_par = self._bbuf_exprs()
    self.w(f'if ({free_cond} && !tfb_tc::mbar_wait(&bars[{BAR_BFREE} + {bsel}], {free_par}, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 71u); }}')
    self._split(NS, bsel)
    self.w('tfb_tc::fence_proxy_async();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{BAR_BFULL} + {bsel}]);')
    self.w(f'tfb_tc::named_sync(2, {NS});   // the raw stage has been read')
    self.open('if (has_next)')
    self._load_b('ntile', NS)
    self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
    if has_r:
      self.w(f'const unsigned nr = (it + 1u) % {nrb}u;')
      self.w(f'// the epilogue of tile it + 1 - {nrb} released this R buffer')
      self.w(f'if (it + 1u >= {nrb}u && !tfb_tc::mbar_wait(&bars[{BAR_RFREE}] + nr, ((it + 1u - {nrb}u) / {nrb}u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 72u); }}')
      self._load_r('ntile', f'(rbase + nr * {L["r_vals"]}u)', NS)
      self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_RFULL}] + nr);')
    self.w('pending = true;')
    self.close()
    self.close()
    self.w('// loads still in flight after an abort must land before the CTA exits')
    self.w(f'if (pending && !tfb_tc::mbar_wait(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) atomicMax(&tfb_err_{b}, 73u);')
    self.w('tfb_tc::cp_async_wait_all();')
    self.close()

  def _epilogue_team(self, lim, BAR_DFULL, BAR_DFREE, BAR_RFULL, BAR_RFREE):
    """Warps 4-15 (three per TMEM lane quadrant): per tile, wait for its accumulators and R
    values, apply R, release both, combine the lane halves and write the tile back."""
    s, L, b = self.s, self.L, self.base
    te, P, M, N = L['te'], L['P'], L['M'], L['N']
    NE = 384
    G3 = 3
    nrb = L['nrb']
    has_r = bool(L['r_off'])
    blocks = L['blocks']
    hs = L['hsplit']
    per = (te + G3 - 1) // G3
    out = s.out
    vol_o = L['vol_o']
    self.open('else if (warp < 16)')
    self.w('const unsigned etid = threadIdx.x - 128u;')
    self.w('const unsigned quad = warp & 3u, grp = (warp >> 2) - 1u;')
    self.w('const unsigned tl = quad * 32u + lane;')
    self.w('const unsigned half = tl >> 6, row = tl & 63u;')
    self.w('const unsigned lane_addr = tmem + ((quad * 32u) << 16);')
    self.w('unsigned it = 0;')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it)')
    self.w(f'if (tfb_tc::any_sync(3, {NE}, !ok)) break;')
    self.w('const unsigned pb = it & 1u;')
    self.w(f'if (!tfb_tc::mbar_wait(&bars[{BAR_DFULL}] + pb, (it >> 1) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 80u); }}')
    if has_r:
      self.w(f'const unsigned rb = it % {nrb}u;')
      self.w(f'if (!tfb_tc::mbar_wait(&bars[{BAR_RFULL}] + rb, (it / {nrb}u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 81u); }}')
      self.w(f'const float* const rprev = rbase + rb * {L["r_vals"]}u;')
    self.w('tfb_tc::fence_after();')
    for k in range(per):
      self.w(f'float p{k}[{N}];')
      self.w('#pragma unroll')
      self.w(f'for (int j = 0; j < {N}; ++j) p{k}[j] = 0.0f;')
    for g in range(G3):
      self.open(f'{"if" if g == 0 else "else if"} (grp == {g}u)')
      for k in range(per):
        e = g + k * G3
        if e >= te:
          continue
        for blk, (tlo, thi, split) in enumerate(blocks):
          if split:
            self.open(f'if (half == {0 if e < hs else 1}u)')
            self._term_partial(tlo, e, blk, f'p{k}')
            self.close()
          else:
            self.open('if (half == 0u)')
            self._term_partial(tlo, e, blk, f'p{k}')
            self.close()
            self.open('else')
            self._term_partial(thi, e, blk, f'p{k}')
            self.close()
      self.close()
    self.w('tfb_tc::fence_before();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{BAR_DFREE}] + pb);')
    if has_r:
      self.w(f'tfb_tc::mbar_arrive(&bars[{BAR_RFREE}] + rb);')
    self.w(f'const size_t pe0 = tile * {te}u;')
    self.w(f'const unsigned nvalid = (unsigned)((numElements - pe0) < {te}u ? (numElements - pe0) : {te}u);')
    self.w('if (etid == 0) tfb_tc::bulk_wait_read();')
    self.w(f'tfb_tc::named_sync(3, {NE});')
    first_half1_assigns = len(s.terms) == 1
    for phase in (0, 1):
      self.open(f'if (half == {phase}u && row < {M}u)')
      for k in range(per):
        e = f'(grp + {k * G3}u)'
        self.open(f'if ({e} < nvalid)')
        self.w(f'float* const dst = stg + {e} * {vol_o}u + row;')
        if phase == 0:
          cond = '' if not blocks[0][2] else f'if ({e} < {hs}u) '
          self.w(f'{cond}{{ ' + ' '.join(f'dst[{j * M}] = p{k}[{j}];' for j in range(N)) + ' }')
        elif first_half1_assigns:
          self.w(f'if ({e} >= {hs}u) {{ ' + ' '.join(f'dst[{j * M}] = p{k}[{j}];' for j in range(N)) + ' }')
        else:
          self.w('{ ' + ' '.join(f'dst[{j * M}] += p{k}[{j}];' for j in range(N)) + ' }')
        self.close()
      self.close()
      if phase == 1:
        self.w('tfb_tc::fence_proxy_async();   // staged values visible to the bulk store')
      self.w(f'tfb_tc::named_sync(3, {NE});')
    bulk_ok = out.addressing.name == 'STRIDED' and out.element_volume() == vol_o and (vol_o * 4) % 16 == 0
    if bulk_ok:
      self.w(f'float* const obase = {out.name} + pe0 * {out.element_volume()}u + {out.name}_extraOffset;')
      self.w('const bool bulk = flags == nullptr && ((reinterpret_cast<uintptr_t>(obase) & 15u) == 0u);')
      self.open('if (bulk)')
      self.open('if (etid == 0)')
      self.w(f'tfb_tc::bulk_store(obase, stg, nvalid * {vol_o * 4}u);')
      self.close()
      self.close()
      self.open('else')
    else:
      self.open('')
    self._store_elements(out, vol_o, 'etid', NE)
    self.close()
    self.close()
    self.w('if (etid == 0) tfb_tc::bulk_wait();')
    self.close()
