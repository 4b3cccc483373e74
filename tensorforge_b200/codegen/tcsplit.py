"""tcgen05 split-precision generator for shared-left GEMM chains (sm_100a tensor cores).

Computes out_e = sum_t A_t * B_{e,t} * R_{e,t} (the chains of plan.chains) as

    out^T[(e,j), i] = sum_t sum_l U_t[l, (e,j)] * A_t[i, l],   U_t = B_{e,t} * R_{e,t}

i.e. one MMA chain per tile of 128 flat output columns (e, j):
  * M = 128 flat columns (one TMEM lane each), N = rows of out padded to 16,
    K = sum_t K_t (each term padded to the MMA K step);
  * A operand (U^T, per element) lives in tensor memory: lane c's producer thread computes
    column j of U_t = B_e * R_t on CUDA cores (the column program of codegen/colprog.py),
    splits it into hi + lo and writes both with tcgen05.st;
  * B operand (A_t^T, shared) is split once per CTA into hi + lo and kept in shared memory
    in the canonical no-swizzle K-major layout (8x16-byte core matrices);
  * D accumulates in tensor memory in FP32 over the three split products
    hi*hi + hi*lo + lo*hi (the lo*lo term is below FP32 resolution); the producer lane
    then reads its output column with tcgen05.ld and stores it contiguously.

Precisions: 'tf32x3' (kind::tf32: hi = value with the 13 low mantissa bits cleared, so
it is exact in TF32, lo = value - hi), 'bf16x3' (kind::f16 with BF16 inputs: hi =
bf16(value), lo = bf16(value - hi)). TF32x3 keeps ~22 significant bits per product;
BF16x3 keeps ~16 (relative error ~1e-5, reported, not used where 1e-6 is required).

Pipelining: A has one TMEM slot per term and D two buffers; mbarriers hand slots between
the 4 producer warps and the MMA-issuing thread, so the tensor cores work on tile n while
the producers compute tile n+1 and store tile n-1. Every mbarrier wait is bounded: on
timeout the kernel records an error code (read with tfb_kernel_error_<name>) and exits
after releasing its tensor memory.
"""
from .. import plan as _plan
from ..plan import Plan
from ..plan.chains import match_left_chain, a_values, r_slots

KSTEP = {'tf32x3': 8, 'bf16x3': 16}
ESIZE = {'tf32x3': 4, 'bf16x3': 2}


def _pad(x, m):
  return (x + m - 1) // m * m


def layout(shape, precision):
  ks = KSTEP[precision]
  es = ESIZE[precision]
  n_mma = _pad(shape.M, 16)
  kpad = [_pad(t.K, ks) for t in shape.terms]
  a_cols = [kp * es // 4 for kp in kpad]          # TMEM columns per split per term
  slot_cols = [2 * c for c in a_cols]               # hi + lo
  tmem_used = sum(slot_cols) + 2 * n_mma
  b_bytes = sum(2 * n_mma * kp * es for kp in kpad)  # hi + lo, all terms
  return dict(ks=ks, es=es, n_mma=n_mma, kpad=kpad, a_cols=a_cols, slot_cols=slot_cols,
              tmem_used=tmem_used, b_bytes=b_bytes)


def plan(chain, shape, precision, variant):
  if precision not in KSTEP:
    return None
  if shape.M > 256:
    return None
  lay = layout(shape, precision)
  if lay['tmem_used'] > 512:
    return None
  chunk = variant.get('chunk', 16 if precision == 'tf32x3' else 16)
  smem = lay['b_bytes'] + 4096 + 8 * (sum(sum(len(c) for c in r_slots(t)) for t in shape.terms if t.R is not None) + shape.N * len(shape.terms))
  smem = max(smem, 120 * 1024)  # one CTA per SM: it owns the SM's tensor memory
  if smem > _plan.SMEM_LIMIT:
    return None
  return Plan('tcsplit', {'precision': precision, 'chunk': chunk}, smem, 160,
              note=f'M={shape.M} N={shape.N} terms={len(shape.terms)} tmem={lay["tmem_used"]}')


HELPERS = r'''
#ifndef TFB_TCGEN05_HELPERS
#define TFB_TCGEN05_HELPERS
#include <cuda_bf16.h>
namespace tfb_tc {
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" :: "r"(smem_u32(bar)) : "memory");
}
// bounded wait on phase `parity`; returns false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long limit) {
  unsigned addr = smem_u32(bar);
  for (unsigned long long it = 0; it < limit; ++it) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(addr), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(unsigned* dst_smem, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ uint64_t smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo & 0x3FFFFu) >> 4) << 16;
  d |= (uint64_t)((sbo & 0x3FFFFu) >> 4) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for tcgen05
  return d;                 // base offset 0, no swizzle (layout type 0)
}
__device__ __forceinline__ void mma_tf32(unsigned d_tmem, unsigned a_tmem, uint64_t b_desc, unsigned idesc, unsigned accum) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}"
               :: "r"(d_tmem), "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accum) : "memory");
}
__device__ __forceinline__ void mma_f16(unsigned d_tmem, unsigned a_tmem, uint64_t b_desc, unsigned idesc, unsigned accum) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}"
               :: "r"(d_tmem), "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accum) : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void st_x8(unsigned taddr, const unsigned* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
               :: "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]) : "memory");
}
__device__ __forceinline__ void st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void ld_x8(unsigned taddr, unsigned* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr) : "memory");
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ unsigned tf32_hi_bits(float x) { return __float_as_uint(x) & 0xFFFFE000u; }
}  // namespace tfb_tc
#endif
'''


def emit_tcsplit(chain, plan_, context, base_name, globals_):
  shape = match_left_chain(chain)
  return _TC(chain, shape, plan_, context, base_name).emit(globals_)


class _TC:
  WAIT_LIMIT = 1 << 26

  def __init__(self, chain, shape, plan_, ctx, base):
    self.chain = chain
    self.s = shape
    self.plan = plan_
    self.ctx = ctx
    self.base = base
    self.prec = plan_.params['precision']
    self.lay = layout(shape, self.prec)
    self.LC = plan_.params['chunk']
    self.H = plan_.params.get('groups', 4)
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

  def _base(self, op, var):
    const = 'const ' if op.is_const else ''
    a = op.addressing.name
    if a == 'STRIDED':
      self.w(f'{const}float* const {var} = {op.name} + e * {op.element_volume()}u + {op.name}_extraOffset;')
    elif a == 'PTR_BASED':
      self.w(f'{const}float* const {var} = {op.name}[e] + {op.name}_extraOffset;')
    else:
      self.w(f'{const}float* const {var} = {op.name};')

  def emit(self, globals_):
    s, lay, b = self.s, self.lay, self.base
    kname = f'kernel_{b}'
    prec = self.prec
    n_mma = lay['n_mma']
    es = lay['es']
    # ---------------------------------------------------------------- tables
    # B operand (A_t^T): for every term, rows i (N, padded to n_mma) x K (padded), hi+lo,
    # canonical no-swizzle K-major layout: (n/8)*SBO + (k/ke)*LBO + (n%8)*16 + (k%ke)*es
    ke = 16 // es
    b_off = []     # byte offset of (term, split) blocks in shared memory
    off = 0
    for ti, kp in enumerate(lay['kpad']):
      b_off.append((off, off + n_mma * kp * es))
      off += 2 * n_mma * kp * es
    b_total = off
    # gather table: for every (term, n, k) dense element, its storage position in A_t (or -1)
    gathers = []
    for ti, t in enumerate(s.terms):
      kp = lay['kpad'][ti]
      look = t.A.sparse_lookup() if t.A.sparse else None
      tbl = []
      for n in range(n_mma):
        for k in range(kp):
          if n < t.A.shape[0] and k < t.K:
            if look is None:
              tbl.append(k * t.A.shape[0] + n)
            else:
              tbl.append(look.get((n, k), -1))
          else:
            tbl.append(-1)
      gathers.append(tbl)
    hdr, pairs, slot_hdr, slot_max = [], [], [], []
    for t in s.terms:
      if t.R is None:
        slot_hdr.append(-1)
        slot_max.append(0)
        continue
      sl = r_slots(t)
      slot_hdr.append(len(hdr))
      slot_max.append(max(len(c) for c in sl))
      for j in range(s.N):
        hdr.append((len(pairs), len(sl[j])))
        for m, pos in sl[j]:
          pairs.append((m * t.K, pos))

    self.w(HELPERS)
    self.w(f'// generated by tensorforge_b200 (strategy: tcsplit, {prec}, chunk={self.LC})')
    self.w('// meta data:')
    for o in self.chain.operands:
      self.w(f'// {o.tensor.gen_descr()}')
    for st in self.chain.stages:
      self.w(f'// {st.descr}')
    for ti, tbl in enumerate(gathers):
      self.w(f'__device__ const short bgather{ti}_{b}[{len(tbl)}] = {{{", ".join(str(x) for x in tbl)}}};')
    if hdr:
      self.w(f'__device__ const int2 shdr_{b}[{len(hdr)}] = {{{", ".join(f"{{{x},{c}}}" for x, c in hdr)}}};')
      self.w(f'__device__ const int2 spair_{b}[{max(1, len(pairs))}] = {{{", ".join(f"{{{x},{c}}}" for x, c in pairs) or "{0,0}"}}};')
    self.w(f'__device__ __align__(16) const float zeros_{b}[{max(self.LC, 16) + 4}] = {{}};')
    self.w(f'__device__ unsigned tfb_err_{b} = 0u;')
    self.w(f'extern "C" int tfb_kernel_error_{b}(void* stream) {{')
    self.w('  unsigned v = 0, z = 0;')
    self.w('  cudaStream_t st = static_cast<cudaStream_t>(stream);')
    self.w(f'  cudaMemcpyFromSymbolAsync(&v, tfb_err_{b}, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);')
    self.w(f'  cudaMemcpyToSymbolAsync(tfb_err_{b}, &z, sizeof(unsigned), 0, cudaMemcpyHostToDevice, st);')
    self.w('  cudaStreamSynchronize(st);')
    self.w('  return (int)v;')
    self.w('}')
    # instruction descriptor: D f32, A/B tf32 (2) or bf16 (1), both K-major, N>>3, M>>4
    fmt = 2 if prec == 'tf32x3' else 1
    idesc = (1 << 4) | (fmt << 7) | (fmt << 10) | ((n_mma >> 3) << 17) | ((128 >> 4) << 24)
    hdr_bytes = 8 * (len(hdr) + len(pairs))
    bar_off = b_total + hdr_bytes
    bar_off = (bar_off + 15) // 16 * 16
    nterms = len(s.terms)
    smem = max(self.plan.smem_bytes, bar_off + 16 * (2 * nterms + 4) + 64)
    self.plan.smem_bytes = smem
    # TMEM column map: slot t = [hi | lo], then D0, D1
    slot_base = []
    col = 0
    for ti in range(nterms):
      slot_base.append(col)
      col += lay['slot_cols'][ti]
    d_base = [col, col + n_mma]
    lim = self.WAIT_LIMIT

    H = self.H
    nthreads = 32 * (4 * H + 1)
    self.w(f'__global__ void __launch_bounds__({nthreads}, 1) {kname}({", ".join(self.params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(1024) unsigned char tfb_smem_raw[];')
    self.w(f'uint64_t* const bars = reinterpret_cast<uint64_t*>(tfb_smem_raw + {bar_off});')
    self.w(f'// bars[0..{nterms}) afull[t], bars[{nterms}..{2 * nterms}) afree[t], bars[{2 * nterms}], [{2 * nterms + 1}] dfull[0/1]')
    self.w(f'unsigned* const tmem_slot = reinterpret_cast<unsigned*>(bars + {2 * nterms + 2});')
    self.w(f'int2* const sHdr = reinterpret_cast<int2*>(tfb_smem_raw + {b_total});')
    self.w(f'int2* const sPair = sHdr + {len(hdr)};')
    self.w('const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;')
    self.w(f'const size_t totalCols = numElements * {s.N}u;')
    self.w('const size_t numTiles = (totalCols + 127u) / 128u;')
    # ---- setup: B operand split into smem, slot tables, barriers, TMEM
    for ti, t in enumerate(s.terms):
      kp = lay['kpad'][ti]
      nvals = n_mma * kp
      hi_off, lo_off = b_off[ti]
      sbo = (kp // ke) * 128
      self.open(f'for (int q = threadIdx.x; q < {nvals}; q += blockDim.x)')
      self.w(f'const int n = q / {kp}, k = q - n * {kp};')
      self.w(f'const int src = bgather{ti}_{b}[q];')
      self.w(f'const float v = src >= 0 ? {t.A.name}[src] : 0.0f;')
      self.w(f'const unsigned boff = (n >> 3) * {sbo}u + (k / {ke}) * 128u + (n & 7) * 16u + (k % {ke}) * {es}u;')
      if prec == 'tf32x3':
        self.w('const unsigned hb = tfb_tc::tf32_hi_bits(v);')
        self.w('const float lo = v - __uint_as_float(hb);')
        self.w(f'*reinterpret_cast<unsigned*>(tfb_smem_raw + {hi_off} + boff) = hb;')
        self.w(f'*reinterpret_cast<float*>(tfb_smem_raw + {lo_off} + boff) = lo;')
      else:
        self.w('const __nv_bfloat16 h = __float2bfloat16_rn(v);')
        self.w('const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));')
        self.w(f'*reinterpret_cast<__nv_bfloat16*>(tfb_smem_raw + {hi_off} + boff) = h;')
        self.w(f'*reinterpret_cast<__nv_bfloat16*>(tfb_smem_raw + {lo_off} + boff) = l;')
      self.close()
    if hdr:
      self.w(f'for (int q = threadIdx.x; q < {len(hdr)}; q += blockDim.x) sHdr[q] = shdr_{b}[q];')
      self.w(f'for (int q = threadIdx.x; q < {len(pairs)}; q += blockDim.x) sPair[q] = spair_{b}[q];')
    self.open('if (threadIdx.x == 0)')
    for ti in range(nterms):
      self.w(f'tfb_tc::mbar_init(&bars[{ti}], {128 * H}u);')
      self.w(f'tfb_tc::mbar_init(&bars[{nterms + ti}], 1u);')
    self.w(f'tfb_tc::mbar_init(&bars[{2 * nterms}], 1u);')
    self.w(f'tfb_tc::mbar_init(&bars[{2 * nterms + 1}], 1u);')
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
    # ---- MMA issuer: warp 4, one thread
    self.open(f'if (warp == {4 * H})')
    self.open('if (lane == 0)')
    self.w('unsigned it = 0;')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles && ok; tile += gridDim.x, ++it)')
    self.w(f'const unsigned dcol = (it & 1u) ? {d_base[1]}u : {d_base[0]}u;')
    for ti, t in enumerate(s.terms):
      kp = lay['kpad'][ti]
      ksteps = kp // lay['ks']
      hi_off, lo_off = b_off[ti]
      sbo = (kp // ke) * 128
      acols = lay['a_cols'][ti]
      self.w(f'if (!tfb_tc::mbar_wait(&bars[{ti}], it & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, {10 + ti}u); break; }}')
      self.w('tfb_tc::fence_after();')
      self.open(f'for (int ks = 0; ks < {ksteps}; ++ks)')
      # A from TMEM: hi at slot_base, lo at slot_base + acols; per k step advance K elems -> cols
      cols_per_step = lay['ks'] * es // 4
      self.w(f'const unsigned a_hi = tmem + {slot_base[ti]}u + ks * {cols_per_step}u;')
      self.w(f'const unsigned a_lo = a_hi + {acols}u;')
      self.w(f'const unsigned b_hi_addr = tfb_tc::smem_u32(tfb_smem_raw + {hi_off}) + ks * 256u;')
      self.w(f'const unsigned b_lo_addr = tfb_tc::smem_u32(tfb_smem_raw + {lo_off}) + ks * 256u;')
      self.w(f'const uint64_t bh = tfb_tc::smem_desc(b_hi_addr, 128u, {sbo}u);')
      self.w(f'const uint64_t bl = tfb_tc::smem_desc(b_lo_addr, 128u, {sbo}u);')
      mma = 'mma_tf32' if prec == 'tf32x3' else 'mma_f16'
      first = '(ks > 0) ? 1u : 0u' if ti == 0 else '1u'
      self.w(f'tfb_tc::{mma}(tmem + dcol, a_hi, bh, {idesc}u, {first});')
      self.w(f'tfb_tc::{mma}(tmem + dcol, a_hi, bl, {idesc}u, 1u);')
      self.w(f'tfb_tc::{mma}(tmem + dcol, a_lo, bh, {idesc}u, 1u);')
      self.close()
      self.w(f'tfb_tc::mma_commit(&bars[{nterms + ti}]);')
    self.w(f'tfb_tc::mma_commit(&bars[{2 * nterms} + (it & 1u)]);')
    self.close()
    self.close()
    self.close()
    # ---- producers / epilogue: warps 0-3, lane = TMEM lane = flat column within the tile
    self.open(f'else if (warp < {4 * H})')
    self.w('const unsigned quad = warp & 3u, grp = warp >> 2;')
    self.w('const unsigned row = quad * 32u + lane;')
    self.w('const unsigned lane_addr = tmem + ((quad * 32u) << 16);')
    self.w('unsigned it = 0;')
    self.w('size_t prev_tile = 0; bool have_prev = false;')
    self.open('for (size_t tile = blockIdx.x; ; tile += gridDim.x, ++it)')
    self.w('const bool more = tile < numTiles && ok;')
    self.open('if (more)')
    self.w('const size_t c = tile * 128u + row;')
    self.w('const bool valid = c < totalCols;')
    self.w(f'const size_t e = valid ? c / {s.N}u : 0;')
    self.w(f'const int j = valid ? (int)(c - e * {s.N}u) : 0;')
    self.w('const bool active = valid && (flags == nullptr || flags[e] != 0u);')
    for ti, t in enumerate(s.terms):
      self._produce_term(ti, t, slot_base[ti], lim)
    self.close()
    # epilogue of the previous tile
    self.open('if (have_prev && ok)')
    self.w(f'const unsigned pb = ((it - 1u) & 1u);')
    self.w(f'if (!tfb_tc::mbar_wait(&bars[{2 * nterms} + pb], ((it - 1u) >> 1) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 20u); }}')
    self.open('if (ok)')
    self.w('tfb_tc::fence_after();')
    self._epilogue(d_base)
    self.close()
    self.close()
    self.w('if (!more) break;')
    self.w('prev_tile = tile; have_prev = true;')
    self.close()
    self.close()
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
    launch = {'kernel': kname, 'block': nthreads, 'elements_per_block': 1, 'smem': smem, 'args': args,
              'grid': f'(numElements * {s.N}u + 127u) / 128u', 'pre': pre}
    return kernel, launch, ''

  # ------------------------------------------------------------------ producer
  def _produce_term(self, ti, t, slot_col, lim):
    b, LC = self.base, self.LC
    lay = self.lay
    prec = self.prec
    es = lay['es']
    kp = lay['kpad'][ti]
    acols = lay['a_cols'][ti]
    nterms = len(self.s.terms)
    self.w(f'// term {ti}: U_{ti} column j -> tensor memory slot {ti} (hi at +0, lo at +{acols})')
    self.open('')
    # wait until the MMAs of the previous tile have finished reading this slot
    self.w(f'if (it > 0 && !tfb_tc::mbar_wait(&bars[{nterms + ti}], (it - 1u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, {30 + ti}u); }}')
    self.w('tfb_tc::fence_after();')
    self._base(t.B, 'pB')
    ms = 0
    if t.R is not None:
      sl = r_slots(t)
      ms = max(len(c) for c in sl)
      self._base(t.R, 'pR')
      self.w(f'const int2 hdr = active ? sHdr[{self._slot_hdr(ti)} + j] : make_int2(0, 0);')
      for q in range(ms):
        self.w(f'const int2 pr{q} = sPair[hdr.x + ({q} < hdr.y ? {q} : 0)];')
        self.w(f'const float* const col{q} = ({q} < hdr.y) ? pB + pr{q}.x : zeros_{b};')
        self.w(f'const float r{q} = ({q} < hdr.y) ? __ldg(pR + pr{q}.y) : 0.0f;')
    for ci, l0 in enumerate(range(0, kp, LC)):
      n = min(LC, kp - l0)
      real = max(0, min(n, t.K - l0))
      self.open(f'if (grp == {ci % self.H}u)')
      self.w(f'float u[{n}];')
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {n}; ++i) u[i] = 0.0f;')
      if real > 0:
        if t.R is None:
          self.open('if (active)')
          self.w('#pragma unroll')
          self.w(f'for (int i = 0; i < {real}; ++i) u[i] = __ldg(pB + (size_t)j * {t.K} + {l0} + i);')
          self.close()
        else:
          for q in range(ms):
            self.w('#pragma unroll')
            self.w(f'for (int i = 0; i < {real}; ++i) u[i] = fmaf(r{q}, __ldg(col{q} + ({q} < hdr.y ? {l0} + i : i)), u[i]);')
      # split and store hi/lo into TMEM (lane = row)
      if prec == 'tf32x3':
        self.w(f'unsigned hv[{n}], lv[{n}];')
        self.w('#pragma unroll')
        self.w(f'for (int i = 0; i < {n}; ++i) {{ hv[i] = tfb_tc::tf32_hi_bits(u[i]); lv[i] = __float_as_uint(u[i] - __uint_as_float(hv[i])); }}')
        for c8 in range(0, n, 8):
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + l0 + c8}u, hv + {c8});')
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols + l0 + c8}u, lv + {c8});')
      else:
        half = n // 2
        self.w(f'unsigned hv[{half}], lv[{half}];')
        self.w('#pragma unroll')
        self.open(f'for (int i = 0; i < {half}; ++i)')
        self.w('const __nv_bfloat16 h0 = __float2bfloat16_rn(u[2 * i]), h1 = __float2bfloat16_rn(u[2 * i + 1]);')
        self.w('const __nv_bfloat16 l0_ = __float2bfloat16_rn(u[2 * i] - __bfloat162float(h0));')
        self.w('const __nv_bfloat16 l1_ = __float2bfloat16_rn(u[2 * i + 1] - __bfloat162float(h1));')
        self.w('hv[i] = (unsigned)__bfloat16_as_ushort(h0) | ((unsigned)__bfloat16_as_ushort(h1) << 16);')
        self.w('lv[i] = (unsigned)__bfloat16_as_ushort(l0_) | ((unsigned)__bfloat16_as_ushort(l1_) << 16);')
        self.close()
        for c8 in range(0, half, 8):
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + l0 // 2 + c8}u, hv + {c8});')
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols + l0 // 2 + c8}u, lv + {c8});')
      self.close()
    self.w('tfb_tc::st_wait();')
    self.w('tfb_tc::fence_before();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{ti}]);')
    self.close()

  def _slot_hdr(self, ti):
    off = 0
    for k, t in enumerate(self.s.terms):
      if k == ti:
        return off
      if t.R is not None:
        off += self.s.N
    return off

  def _epilogue(self, d_base):
    s = self.s
    M = s.M
    nld = (M + 7) // 8
    H = self.H
    self.w(f'const unsigned dcol = pb ? {d_base[1]}u : {d_base[0]}u;')
    per = (nld + H - 1) // H
    self.w(f'unsigned dv[{per * 8}];')
    for k in range(per):
      # group g loads x8 block q = g + k*H (clamped; the duplicate is not stored)
      self.w(f'tfb_tc::ld_x8(lane_addr + dcol + 8u * (grp + {k * H}u < {nld}u ? grp + {k * H}u : 0u), dv + {8 * k});')
    self.w('tfb_tc::ld_wait();')
    self.w('const size_t c = prev_tile * 128u + row;')
    self.open('if (c < totalCols)')
    self.w(f'const size_t e = c / {s.N}u;')
    self.w(f'const int j = (int)(c - e * {s.N}u);')
    self.open('if (flags == nullptr || flags[e] != 0u)')
    self._base(s.out, 'pO')
    self.w(f'float* const col = pO + (size_t)j * {M};')
    for k in range(per):
      self.w(f'const unsigned q{k} = grp + {k * H}u;')
      self.open(f'if (q{k} < {nld}u)')
      self.w(f'float* const dst = col + 8u * q{k};')
      last = M - 8 * (nld - 1)
      self.w(f'const unsigned cnt = (q{k} == {nld - 1}u) ? {last}u : 8u;')
      if s.accumulate:
        self.w(f'for (unsigned i = 0; i < cnt; ++i) dst[i] += __uint_as_float(dv[{8 * k} + i]);')
      else:
        self.open('if (cnt == 8u && (reinterpret_cast<uintptr_t>(dst) & 15u) == 0u)')
        self.w(f'reinterpret_cast<float4*>(dst)[0] = make_float4(__uint_as_float(dv[{8*k}]), __uint_as_float(dv[{8*k+1}]), __uint_as_float(dv[{8*k+2}]), __uint_as_float(dv[{8*k+3}]));')
        self.w(f'reinterpret_cast<float4*>(dst)[1] = make_float4(__uint_as_float(dv[{8*k+4}]), __uint_as_float(dv[{8*k+5}]), __uint_as_float(dv[{8*k+6}]), __uint_as_float(dv[{8*k+7}]));')
        self.close()
        self.open('else')
        self.w(f'for (unsigned i = 0; i < cnt; ++i) dst[i] = __uint_as_float(dv[{8 * k} + i]);')
        self.close()
      self.close()
    self.close()
    self.close()
