"""Column-program generator (CUDA cores) for shared-left GEMM chains.

Computes out_e = sum_t A_t * B_{e,t} * R_{e,t} (plan/chains.py) on CUDA cores, tile by
tile, a tile being TE whole elements (TE*N flat output columns (e, j)):

  1. U phase: one thread per (element, row l) reads row l of B_{e,t} with coalesced
     loads (consecutive threads -> consecutive rows), multiplies it by R_{e,t} with R's
     compile-time pattern unrolled (only its nonzeros cost an FMA) and writes row l of
     U_t = B_{e,t} * R_{e,t} into a padded shared-memory buffer (pitch = K + 4 floats,
     so that the column reads of step 2 are bank-conflict free).
  2. K stage: one thread per flat column reads its column of U_t (16-byte loads) and
     accumulates acc += A_t * u, fully unrolled over A_t's compile-time nonzero pattern.
     A_t's values are FMA operands straight from the constant bank (one copy per module,
     refreshed by the launcher on the launch stream), or, with variant a_source='smem',
     128-bit broadcast loads from shared memory.
  3. The tile's output is staged in shared memory and written back with coalesced
     16-byte stores (or per column when masked, accumulated or pointer-addressed).

Intermediates never leave the SM; B, R and out are touched once per element. The grid is
persistent (SMs x occupancy) and walks the tiles.
The contraction order differs from the reference's (T_t = A_t*B first, then T_t*R_t);
results agree within FP32 rounding (tests hold them to 1e-5 of the output scale).
"""
from ..plan.chains import match_left_chain, a_values


def _pad(x, m):
  return (x + m - 1) // m * m


CP_HELPERS = r'''
#ifndef TFB_CP_ASYNC_HELPERS
#define TFB_CP_ASYNC_HELPERS
namespace tfb_cp {
__device__ __forceinline__ void copy16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void copy4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void copy8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
}  // namespace tfb_cp
#endif
'''


def emit_colprog(chain, plan, context, base_name, globals_):
  shape = match_left_chain(chain)
  return _ColProg(chain, shape, plan, context, base_name).emit(globals_)


def tile_elements(shape, threads, cols=1):
  """Elements per tile: `cols` columns per thread, whole elements of N columns each."""
  return cols * max(1, threads // shape.N)


class _ColProg:
  def __init__(self, chain, shape, plan, ctx, base):
    self.chain = chain
    self.s = shape
    self.plan = plan
    self.ctx = ctx
    self.base = base
    self.T = ctx.fp_as_str()
    self.dbl = self.T == 'double'
    self.FS = 8 if self.dbl else 4
    self.VEC = 2 if self.dbl else 4
    self.VT = 'double2' if self.dbl else 'float4'
    self.FMA = 'fma' if self.dbl else 'fmaf'
    self.BT = plan.params['threads']
    self.LC = plan.params['chunk']
    self.asrc = plan.params.get('a_source', 'const')
    # leading terms whose A values are constant-bank FMA operands; the rest read shared memory
    nterms = len(shape.terms)
    self.const_terms = {'const': nterms, 'smem': 0}.get(self.asrc, int(plan.params.get('const_terms', 0)))
    self.term_const = [ti < self.const_terms for ti in range(nterms)]
    self.prefetch = bool(plan.params.get('prefetch', 1)) and not getattr(self, 'grouped', False)
    self.CPT = int(plan.params.get('cols', 1))
    # row split: RS groups of threads share the tile's columns, group g accumulating rows
    # [g * MR, (g + 1) * MR) of every column it owns (RS x the warps for the same registers)
    self.RS = int(plan.params.get('rsplit', 1))
    self.CT = self.BT // self.RS          # threads per row group (column threads)
    self.TE = tile_elements(shape, self.CT, self.CPT)
    self.TC = self.TE * shape.N
    self.TCT = self.TC // self.CPT        # columns per round: thread t owns t + r * TCT
    self.MR = _pad(-(-shape.M // self.RS), self.VEC) if self.RS > 1 else shape.M
    self.kmax = max(t.K for t in shape.terms)
    # U^T rows: K + VEC values keep 16-byte row starts (vector loads) and spread the rows of
    # a quarter-warp over the banks; an odd pitch (scalar loads) is conflict-free and smaller
    if plan.params.get('upitch', 'vec') == 'odd':
      self.pitch = self.kmax | 1
    else:
      self.pitch = _pad(self.kmax, self.VEC) + self.VEC
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

  def lit(self, v):
    return self.ctx.fp_type.literal(v)

  def block(self, head):
    em = self

    class _B:
      def __enter__(self_):
        em.open(head)

      def __exit__(self_, *a):
        em.close()
    return _B()

  def params(self, globals_):
    params = []
    for t, _ in globals_:
      dt = self.T if t.datatype is None else str(t.datatype)
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

  # ------------------------------------------------------------------ emit
  def _layout(self):
    s = self.s
    # A storage: every term's values, in storage order, concatenated
    self.a_base = []
    ctot = stot = 0
    for ti, t in enumerate(s.terms):
      if self.term_const[ti]:
        self.a_base.append(ctot)
        ctot += t.A.storage_size()
      else:
        self.a_base.append(stot)
        stot += t.A.storage_size()
    self.a_const_total, self.a_smem_total = ctot, stot
    self.a_total = ctot + stot
    # rounded to whole vectors: the staged R copies behind it are read as float4 / double2
    self.ubuf_vals = _pad(max(self.TC * self.pitch, self.TC * s.M), self.VEC)
    # per-tile copies of the batched R operands (read as 128-bit broadcast loads)
    # (not needed with the prefetch stage, which holds them)
    self.r_off = {}
    r_vals = 0
    for t in s.terms:
      if not self.prefetch and t.R is not None and t.R.kind == 'batched' and t.R.name not in self.r_off:
        self.r_off[t.R.name] = self.ubuf_vals + r_vals
        r_vals += self.TE * _pad(t.R.storage_size(), self.VEC)
    self.work_vals = _pad(self.ubuf_vals + r_vals, self.VEC)   # ubuf + staged R, per CTA
    # prefetch stage: the next tile's batched B / R operands, copied with cp.async while the
    # last K stage of the current tile runs (standalone kernels only)
    self.stage_off, self.stage_vals = {}, 0
    if self.prefetch:
      for t in s.terms:
        for op in (t.B, t.R):
          if op is not None and op.kind == 'batched' and op.name not in self.stage_off:
            self.stage_off[op.name] = self.work_vals + self.stage_vals
            self.stage_vals += self.TE * _pad(op.storage_size() if op.sparse else op.element_volume(), self.VEC)
    a_smem = _pad(self.a_smem_total, self.VEC) if self.a_smem_total else 0
    self.a_off = self.work_vals + self.stage_vals
    self.smem = (self.work_vals + self.stage_vals + a_smem) * self.FS

  def _header(self):
    if self.prefetch:
      self.w(CP_HELPERS)
    self.w(f'// generated by tensorforge_b200 (strategy: colprog, threads={self.BT}, chunk={self.LC}, '
           f'tile={self.TE} elements, A from {self.asrc})')
    self.w('// meta data:')
    for o in self.chain.operands:
      self.w(f'// {o.tensor.gen_descr()}')
    for st in self.chain.stages:
      self.w(f'// {st.descr}')

  def _prefetch(self, tile_expr):
    """cp.async the tile's batched B / R operands into the stage (16-byte chunks when aligned)."""
    T, BT, VEC, FS = self.T, self.BT, self.VEC, self.FS
    ops = {o.name: o for o in self.chain.operands}
    for name, off in self.stage_off.items():
      op = ops[name]
      vals = op.storage_size() if op.sparse else op.element_volume()
      vp = _pad(vals, VEC)
      self.open('')
      self.w(f'const size_t pe0 = ({tile_expr}) * {self.TE}u;')
      small = 'copy8' if FS == 8 else 'copy4'
      if op.addressing.name == 'PTR_BASED':
        # one element per warp at a time: its pointer is loaded once, not once per chunk
        self.open(f'for (unsigned ei = threadIdx.x >> 5; ei < {self.TE}u; ei += {BT // 32}u)')
        self.w('const size_t ee = pe0 + ei;')
        self.w('if (ee >= numElements) break;')
        self.w(f'const {T}* const sbase = {self._elem_ptr(op, "ee")};')
        self.w(f'{T}* const dbase = ubuf + {off} + ei * {vp}u;')
        if vals % VEC == 0:
          self.w('const bool al = (reinterpret_cast<uintptr_t>(sbase) & 15u) == 0u;')
          self.open(f'for (unsigned c = threadIdx.x & 31u; c < {vals // VEC}u; c += 32u)')
          self.w(f'const {T}* src = sbase + {VEC}u * c;')
          self.w(f'{T}* dst = dbase + {VEC}u * c;')
          self.w('if (al) tfb_cp::copy16(dst, src);')
          self.w('else { ' + ' '.join(f'tfb_cp::{small}(dst + {i}, src + {i});' for i in range(VEC)) + ' }')
          self.close()
        else:
          self.w(f'for (unsigned c = threadIdx.x & 31u; c < {vals}u; c += 32u) tfb_cp::{small}(dbase + c, sbase + c);')
        self.close()
      elif vals % VEC == 0:
        self.open(f'for (unsigned q = threadIdx.x; q < {self.TE * vals // VEC}u; q += {BT}u)')
        self.w(f'const unsigned ei = q / {vals // VEC}u, c = q - ei * {vals // VEC}u;')
        self.w('const size_t ee = pe0 + ei;')
        self.open('if (ee < numElements)')
        self.w(f'const {T}* src = {self._elem_ptr(op, "ee")} + {VEC}u * c;')
        self.w(f'{T}* dst = ubuf + {off} + ei * {vp}u + {VEC}u * c;')
        self.w('if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0u) tfb_cp::copy16(dst, src);')
        self.w('else { ' + ' '.join(f'tfb_cp::{small}(dst + {i}, src + {i});' for i in range(VEC)) + ' }')
        self.close()
        self.close()
      else:
        self.open(f'for (unsigned q = threadIdx.x; q < {self.TE * vals}u; q += {BT}u)')
        self.w(f'const unsigned ei = q / {vals}u, c = q - ei * {vals}u;')
        self.w('const size_t ee = pe0 + ei;')
        self.w(f'if (ee < numElements) tfb_cp::{small}(ubuf + {off} + ei * {vp}u + c, {self._elem_ptr(op, "ee")} + c);')
        self.close()
      self.close()

  def _tile_body(self):
    """Code for one tile; expects `tile`, `ubuf`, (`sA`), the ABI names, numElements, flags."""
    s, T, BT = self.s, self.T, self.BT
    if self.RS > 1:
      self.w(f'const unsigned ct = threadIdx.x % {self.CT}u, rg = threadIdx.x / {self.CT}u;')
    else:
      self.w('const unsigned ct = threadIdx.x;')
    self.w(f'const unsigned le = ct / {s.N}u, lj = ct - le * {s.N}u;')
    self.w(f'const size_t e0 = tile * {self.TE}u;')
    for r in range(self.CPT):
      sfx = '' if r == 0 else str(r)
      self.w(f'const size_t el{sfx} = e0 + le + {r * (self.TCT // s.N)}u;')
      self.w(f'const bool lane_ok{sfx} = ct < {self.TCT}u && el{sfx} < numElements;')
      self.w(f'const bool active{sfx} = lane_ok{sfx} && (flags == nullptr || flags[el{sfx}] != 0u);')
    for name, off in ([] if self.prefetch else self.r_off.items()):
      op = [o for o in self.chain.operands if o.name == name][0]
      nr = op.storage_size()
      nrp = _pad(nr, self.VEC)
      self.open(f'for (unsigned q = threadIdx.x; q < {self.TE * nr}u; q += {BT}u)')
      self.w(f'const unsigned ei = q / {nr}u, p = q - ei * {nr}u;')
      self.w('const size_t e = e0 + ei;')
      self.w(f'ubuf[{off} + ei * {nrp}u + p] = e < numElements ? __ldg({self._elem_ptr(op, "e")} + p) : {self.lit(0)};')
      self.close()
    if self.r_off and not self.prefetch:
      self.w('__syncthreads();')
    for r in range(self.CPT):
      a = 'acc' if r == 0 else f'acc{r}'
      self.w(f'{T} {a}[{self.MR}];')
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {self.MR}; ++i) {a}[i] = {self.lit(0)};')
    for ti, t in enumerate(s.terms):
      self._term(ti, t)
    self._epilogue()
    self._store()

  def emit(self, globals_):
    s = self.s
    T, BT = self.T, self.BT
    b = self.base
    kname = f'kernel_{b}'
    self._layout()
    self._header()
    if self.a_const_total:
      self.w(f'__constant__ {T} cA_{b}[{self.a_const_total}];')
    mb = self.plan.params.get('min_blocks', 0)
    bounds = f'{BT}, {mb}' if mb else f'{BT}'
    self.w(f'__global__ void __launch_bounds__({bounds}) {kname}({", ".join(self.params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(16) unsigned char tfb_smem_raw[];')
    self.w(f'{T}* const ubuf = reinterpret_cast<{T}*>(tfb_smem_raw);')
    if self.a_smem_total:
      self.w(f'{T}* const sA = ubuf + {self.a_off};')
      for ti, t in enumerate(s.terms):
        if not self.term_const[ti]:
          self.w(f'for (int q = threadIdx.x; q < {t.A.storage_size()}; q += {BT}) sA[{self.a_base[ti]} + q] = {t.A.name}[q];')
      self.w('__syncthreads();')
    self.w(f'const size_t numTiles = (numElements + {self.TE - 1}u) / {self.TE}u;')
    if self.prefetch:
      self.w('if (blockIdx.x < numTiles) {')
      self.ind += 1
      self._prefetch('(size_t)blockIdx.x')
      self.ind -= 1
      self.w('}')
      self.w('tfb_cp::commit();')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x)')
    if self.prefetch:
      self.w('tfb_cp::wait_all();')
      self.w('__syncthreads();')
    self._tile_body()
    self.close()
    if self.prefetch:
      self.w('tfb_cp::wait_all();')
    self.ind -= 1
    self.w('}')
    kernel = '\n'.join(self.lines)
    return kernel, self._launch(globals_, kname), ''

  # ------------------------------------------------------------------ grouped launches
  def emit_group_functions(self, globals_, gid):
    """Device functions for one group of a grouped (mixed-shape) launch: A staging and one tile.

    The group's ABI symbols arrive through a tfb_group_args record (pointers, extra offsets,
    element count, flags); A is read from shared memory (staged when the group changes).
    With the plan's prefetch stage the group also gets `group<g>_prefetch` (cp.async of a
    tile's batched inputs into the stage), and its tile function takes the next work item's
    tile when that item belongs to the same group (~0 otherwise) and fetches it during its
    last K stage.
    """
    assert self.asrc == 'smem'
    s, T, BT = self.s, self.T, self.BT
    if self.prefetch:
      self.next_tile = 'next_tile'
    self._layout()
    self._header()
    decl = []
    for i, (t, _) in enumerate(globals_):
      dt = self.T if t.datatype is None else str(t.datatype)
      const = 'const ' if t.direction.name == 'SOURCE' else ''
      ptr = t.addressing.to_pointer()
      decl.append(f'{const}{dt}{ptr} const __restrict__ {t.name} = reinterpret_cast<{const}{dt}{ptr}>(const_cast<void*>(ga.ptr[{i}]));')
      if t.addressing.name != 'NONE':
        decl.append(f'const unsigned {t.name}_extraOffset = ga.off[{i}];')
    self.w(f'__device__ __forceinline__ void group{gid}_stage_a(const tfb_group_args& ga, {T}* sA) {{')
    self.ind += 1
    for d in decl:
      self.w(d)
    for ti, t in enumerate(s.terms):
      self.w(f'for (int q = threadIdx.x; q < {t.A.storage_size()}; q += {BT}) sA[{self.a_base[ti]} + q] = {t.A.name}[q];')
    self.ind -= 1
    self.w('}')
    if self.prefetch:
      self.w(f'__device__ __forceinline__ void group{gid}_prefetch(const tfb_group_args& ga, size_t tile, {T}* ubuf) {{')
      self.ind += 1
      for d in decl:
        self.w(d)
      self.w('const size_t numElements = (size_t)ga.num_elements;')
      self._prefetch('tile')
      self.ind -= 1
      self.w('}')
    nxt = ', size_t next_tile' if self.prefetch else ''
    self.w(f'__device__ __forceinline__ void group{gid}_tile(const tfb_group_args& ga, size_t tile, {T}* ubuf, const {T}* sA{nxt}) {{')
    self.ind += 1
    for d in decl:
      self.w(d)
    self.w('const size_t numElements = (size_t)ga.num_elements;')
    self.w('const unsigned* const flags = ga.flags;')
    if self.prefetch:
      self.w('tfb_cp::wait_all();  // this tile\'s stage has landed')
      self.w('__syncthreads();')
    self._tile_body()
    self.ind -= 1
    self.w('}')
    return '\n'.join(self.lines)

  def _launch(self, globals_, kname):
    s, BT, b = self.s, self.BT, self.base
    args = []
    for t, _ in globals_:
      args.append(t.name)
      if t.addressing.name not in ('NONE', 'SCALAR'):
        args.append(f'{t.name}_extraOffset')
    args += ['numElements', 'flags']
    pre = [f'  static int occ[64];',
           f'  if (device < 64 && occ[device] == 0) {{',
           f'    int sms = 0, per = 0;',
           f'    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);',
           f'    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, {kname}, {BT}, {self.smem});',
           f'    occ[device] = (per > 0 ? per : 1) * (sms > 0 ? sms : 1);',
           f'  }}',
           f'  const size_t cap = device < 64 ? (size_t)occ[device] : (size_t)1024;',
           f'  if (grid.x > cap) grid.x = (unsigned)cap;']
    if self.a_const_total:
      # the constant bank is one per module: refresh it on the launch stream, and order
      # launches issued from different streams after the previous launch (outside capture)
      pre += [f'  static std::mutex mu;',
              f'  static cudaEvent_t lastEv[64];',
              f'  static cudaStream_t lastStream[64];',
              f'  static bool haveLast[64];',
              f'  std::lock_guard<std::mutex> guard(mu);',
              f'  cudaStreamCaptureStatus cap_status = cudaStreamCaptureStatusNone;',
              f'  cudaStreamIsCapturing(stream, &cap_status);',
              f'  const bool capturing = cap_status != cudaStreamCaptureStatusNone;',
              f'  if (!capturing && device < 64 && haveLast[device] && lastStream[device] != stream)',
              f'    cudaStreamWaitEvent(stream, lastEv[device], 0);']
      for ti, t in enumerate(s.terms):
        if self.term_const[ti]:
          pre.append(f'  cudaMemcpyToSymbolAsync(cA_{b}, {t.A.name}, {t.A.storage_size() * self.FS}, '
                     f'{self.a_base[ti] * self.FS}, cudaMemcpyDeviceToDevice, stream);')
      pre += [f'  {kname}<<<grid, block, {self.smem}, stream>>>({", ".join(args)});',
              f'  CHECK_ERR;',
              f'  if (!capturing && device < 64) {{',
              f'    if (!haveLast[device]) cudaEventCreateWithFlags(&lastEv[device], cudaEventDisableTiming);',
              f'    cudaEventRecord(lastEv[device], stream);',
              f'    lastStream[device] = stream;',
              f'    haveLast[device] = true;',
              f'  }}']
    self.plan.smem_bytes = self.smem
    return {'kernel': kname, 'block': BT, 'elements_per_block': self.TE, 'smem': self.smem, 'args': args,
            'grid': f'(numElements + {self.TE - 1}u) / {self.TE}u', 'pre': '\n'.join(pre),
            'launched': bool(self.a_const_total)}

  # ------------------------------------------------------------------ pieces
  def _term(self, ti, t):
    s = self.s
    T, BT, VEC, VT, FMA, LC = self.T, self.BT, self.VEC, self.VT, self.FMA, self.LC
    b = self.base
    P, K = t.P, t.K
    pitch = self.pitch
    self.w(f'// term {ti}: A={t.A.name} ({t.A.shape[0]}x{t.A.shape[1]}, {"sparse" if t.A.sparse else "dense"}), '
           f'B={t.B.name}, R={t.R.name if t.R is not None else "-"}')
    # U phase: thread (group g, row l) with l = tid % KP2 computes row l of U_t for the
    # elements g, g + groups, ... (compile-time trip count, loads of all elements in flight)
    kp2 = 1
    while kp2 < K:
      kp2 *= 2
    groups = max(1, BT // kp2)
    per = (self.TE + groups - 1) // groups
    self.open('')
    self.w(f'const unsigned l = threadIdx.x & {kp2 - 1}u, g = threadIdx.x / {kp2}u;')
    self.w('#pragma unroll')
    self.open(f'for (unsigned k = 0; k < {per}u; ++k)')
    self.w(f'const unsigned ei = g + k * {groups}u;')
    self.w('const size_t e = e0 + ei;')
    self.open(f'if (l < {K}u && ei < {self.TE}u && e < numElements)')
    self.w(f'{T}* const urow = ubuf + ei * {s.N * pitch}u + l;')
    if self.prefetch:
      bv = _pad(t.B.element_volume(), VEC)
      self.w(f'const {T}* const bq = ubuf + {self.stage_off[t.B.name]} + ei * {bv}u + l;')
      ld = lambda x: f'bq[{x}]'
    else:
      self.w(f'const {T}* const bq = {self._elem_ptr(t.B, "e")} + l;')
      ld = lambda x: f'__ldg(bq + {x})'
    if t.R is None:
      for j in range(s.N):
        self.w(f'urow[{j * pitch}] = {ld(j * K)};')
    else:
      for m in range(P):
        self.w(f'const {T} q{m} = {ld(m * K)};')
      nr = t.R.storage_size()
      comps = ['x', 'y', 'z', 'w'][:VEC]
      if t.R.kind == 'batched':
        nrp = _pad(nr, VEC)
        roff = self.stage_off[t.R.name] if self.prefetch else self.r_off[t.R.name]
        self.w(f'const {VT}* const rq = reinterpret_cast<const {VT}*>(ubuf + {roff} + ei * {nrp}u);')
        for v in range((nr + VEC - 1) // VEC):
          self.w(f'const {VT} r{v} = rq[{v}];')
        rv = lambda pos: f'r{pos // VEC}.{comps[pos % VEC]}'
      else:
        rv = lambda pos: f'__ldg({t.R.name} + {pos})'
      look = t.R.sparse_lookup() if t.R.sparse else None
      for j in range(s.N):
        expr = self.lit(0)
        for m in range(P):
          pos = look.get((m, j)) if look is not None else j * P + m
          if pos is not None:
            expr = f'{FMA}(q{m}, {rv(pos)}, {expr})'
        self.w(f'urow[{j * pitch}] = {expr};')
    self.close()
    self.close()
    self.close()
    self.w('__syncthreads();')
    if self.prefetch and ti == len(s.terms) - 1:
      self.w('// the stage is free: fetch the next tile while this K stage runs')
      if getattr(self, 'next_tile', None) is None:
        self.open('if (tile + gridDim.x < numTiles)')
        self._prefetch('tile + gridDim.x')
      else:
        # grouped launch: the next work item when it belongs to the same group
        self.open(f'if ({self.next_tile} != ~(size_t)0)')
        self._prefetch(self.next_tile)
      self.close()
      self.w('tfb_cp::commit();')
    # K stage: each A value is an FMA operand for every column the thread owns
    R = range(self.CPT)
    sfx = lambda r: '' if r == 0 else str(r)
    self.open('if (' + ' || '.join(f'active{sfx(r)}' for r in R) + ')')
    for r in R:
      self.w(f'const {T}* const ucol{sfx(r)} = ubuf + (ct + {r * self.TCT}u) * {pitch}u;')
    cols = a_values(t)
    comps = ['x', 'y', 'z', 'w'][:VEC]
    for g in range(self.RS):
      r0, r1 = g * self.MR, min(s.M, (g + 1) * self.MR)
      if self.RS > 1:
        self.open(f'if (rg == {g}u)')
      self._k_stage_rows(ti, t, cols, r0, r1, comps)
      if self.RS > 1:
        self.close()
    self.close()
    self.w('__syncthreads();')

  def _k_stage_rows(self, ti, t, cols, r0, r1, comps):
    """Unrolled FMAs of term ti over the nonzeros of A_t in rows [r0, r1) (acc index i - r0)."""
    T, VEC, VT, FMA, LC = self.T, self.VEC, self.VT, self.FMA, self.LC
    b = self.base
    K = t.K
    R = range(self.CPT)
    sfx = lambda r: '' if r == 0 else str(r)
    # shared-memory A is consumed in storage order: fetch it one aligned vector at a time
    # (one broadcast LDS.128 / LDS.64 per VEC values) instead of one load per value
    loaded = set()

    def a_operand(pos):
      if self.term_const[ti]:
        return f'cA_{b}[{self.a_base[ti] + pos}]'
      g = self.a_base[ti] + pos
      v = g // VEC
      if v not in loaded:
        loaded.add(v)
        self.w(f'const {VT} av{v} = reinterpret_cast<const {VT}*>(sA)[{v}];')
      return f'av{v}.{comps[g % VEC]}'
    for l0 in range(0, K, LC):
      n = min(LC, K - l0)
      if not any(r0 <= i < r1 for l in range(l0, l0 + n) for (i, _) in cols[l][1]):
        continue
      self.open('')
      loaded.clear()  # vectors are declared per chunk block
      for r in R:
        u, uc = f'u{sfx(r)}', f'ucol{sfx(r)}'
        self.w(f'{T} {u}[{n}];')
        nv = n // VEC if self.pitch % VEC == 0 else 0
        for v in range(nv):
          self.w(f'{{ const {VT} x = *reinterpret_cast<const {VT}*>({uc} + {l0 + v * VEC}); '
                 + ' '.join(f'{u}[{v * VEC + c}] = x.{comps[c]};' for c in range(VEC)) + ' }')
        for i in range(nv * VEC, n):
          self.w(f'{u}[{i}] = {uc}[{l0 + i}];')
      for l in range(l0, l0 + n):
        for (i, pos) in cols[l][1]:
          if not r0 <= i < r1:
            continue
          a = a_operand(pos)
          if self.CPT == 1:
            self.w(f'acc[{i - r0}] = {FMA}({a}, u[{l - l0}], acc[{i - r0}]);')
          else:
            self.open('')
            self.w(f'const {T} av = {a};')
            for r in R:
              acc = f'acc{sfx(r)}'
              self.w(f'{acc}[{i - r0}] = {FMA}(av, u{sfx(r)}[{l - l0}], {acc}[{i - r0}]);')
            self.close()
      self.close()

  def _epilogue(self):
    """Elementwise stages on the finished output column in registers (row i = n0, the
    thread's column lj = n1), before the store; an accumulated output adds the previous
    value first, so the statements see the chain's final result."""
    s = self.s
    if not s.epilogue:
      return
    from .elementwise import RegisterPointEmitter
    T, M = self.T, s.M
    counter = [0]
    for r in range(self.CPT):
      sf = '' if r == 0 else str(r)
      self.w(f'// elementwise epilogue ({len(s.epilogue)} stage(s)) on column lj of element el{sf}')
      self.open(f'if (active{sf})')
      if s.accumulate:
        self.w(f'const {T}* const prev = {self._elem_ptr(s.out, "el" + sf)} + (size_t)lj * {M}u;')
        self.w('#pragma unroll')
        self.w(f'for (int i = 0; i < {M}; ++i) acc{sf}[i] += prev[i];')
      for st in s.epilogue:
        for i in range(M):
          self.open('')
          pe = RegisterPointEmitter(self, st, s.out, f'acc{sf}', i, 'lj', M,
                                    lambda o, sf=sf: self._elem_ptr(o, 'el' + sf), counter)
          pe.declare_temporaries()
          pe.statements(st.statements)
          self.close()
      self.close()

  def _store(self):
    s = self.s
    T, BT, VEC, VT = self.T, self.BT, self.VEC, self.VT
    o = s.out
    M = s.M
    vol = o.element_volume()
    sfx = lambda r: '' if r == 0 else str(r)
    coalesced = (o.addressing.name == 'STRIDED' and vol == M * s.N and vol % VEC == 0 and M % VEC == 0
                 and not s.accumulate)
    groups = [(g, g * self.MR, min(M, (g + 1) * self.MR)) for g in range(self.RS)]

    def by_group(body):
      for g, r0, r1 in groups:
        if self.RS > 1:
          self.open(f'if (rg == {g}u)')
        body(r0, r1)
        if self.RS > 1:
          self.close()

    def per_column():
      for r in range(self.CPT):
        self.open(f'if (active{sfx(r)})')
        self.w(f'{T}* const col = {self._elem_ptr(o, "el" + sfx(r))} + (size_t)lj * {M}u;')
        op = '+=' if s.accumulate and not s.epilogue else '='

        def body(r0, r1, r=r):
          self.w('#pragma unroll')
          self.w(f'for (int i = {r0}; i < {r1}; ++i) col[i] {op} acc{sfx(r)}[i - {r0}];')
        by_group(body)
        self.close()

    if coalesced:
      self.w('// stage the tile in shared memory, then write it back with coalesced 16-byte stores')
      self.w(f'{T}* const obase = {o.name} + e0 * {vol}u + {o.name}_extraOffset;')
      self.w(f'const bool vec_out = flags == nullptr && ((reinterpret_cast<uintptr_t>(obase) & 15u) == 0u);')
      self.open('if (vec_out)')
      for r in range(self.CPT):
        self.open(f'if (lane_ok{sfx(r)})')

        def body(r0, r1, r=r):
          for v in range(r0 // VEC, r1 // VEC):
            vals = ', '.join(f'acc{sfx(r)}[{v * VEC + c - r0}]' for c in range(VEC))
            self.w(f'reinterpret_cast<{VT}*>(ubuf + (ct + {r * self.TCT}u) * {M}u)[{v}] = make_{VT}({vals});')
        by_group(body)
        self.close()
      self.w('__syncthreads();')
      self.w(f'const size_t nvalid = (numElements - e0) < {self.TE}u ? (numElements - e0) : {self.TE}u;')
      self.w(f'const unsigned nv = (unsigned)(nvalid * {vol // VEC}u);')
      self.w(f'for (unsigned q = threadIdx.x; q < nv; q += {BT}u) '
             f'reinterpret_cast<{VT}*>(obase)[q] = reinterpret_cast<const {VT}*>(ubuf)[q];')
      self.w('__syncthreads();')
      self.close()
      self.open('else')
      per_column()
      self.close()
    else:
      per_column()
