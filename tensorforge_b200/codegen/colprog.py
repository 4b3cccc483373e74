"""Column-program generator (CUDA cores) for shared-left GEMM chains.

One thread computes one output column (e, j) of out_e = sum_t A_t * B_{e,t} * R_{e,t}:

  1. u = column j of V_t = B_{e,t} * R_{e,t}: the nonzeros (m, r) of column j of R_t are
     read up front (unrolled to the pattern's longest column, inactive slots point at a
     zero buffer so the code is branch-free), then u += r * B_{e,t}[rows, m] is
     accumulated chunk by chunk with 16-byte loads of the contiguous column.
  2. acc += A_t * u: fully unrolled over A_t's compile-time nonzero pattern, so only
     nonzeros cost an FFMA. A_t's values are staged once per CTA in shared memory in
     exactly the order the FFMAs consume them and read as 128-bit broadcast loads
     (one load feeds 4 FP32 / 2 FP64 FMAs).
  3. out_e[:, j] (+)= acc, stored as one contiguous column.

Intermediates never leave registers; B, R and out are touched once per element, so
HBM traffic is the algorithmic minimum. The grid is persistent (SMs x occupancy) and
walks the flat column space, so any element count and any N is load balanced. Two
instantiations are emitted: 16-byte vector accesses when every strided operand is
16-byte aligned (checked by the launcher), scalar accesses otherwise.
The contraction order differs from the reference's (T_t = A_t*B first, then T_t*R_t);
results agree within FP32 rounding (tests hold them to 1e-5 of the output scale).
"""
from ..plan.chains import match_left_chain, a_values, r_slots


def emit_colprog(chain, plan, context, base_name, globals_):
  shape = match_left_chain(chain)
  em = _ColProg(chain, shape, plan, context, base_name)
  return em.emit(globals_)


class _ColProg:
  def __init__(self, chain, shape, plan, ctx, base):
    self.chain = chain
    self.s = shape
    self.plan = plan
    self.ctx = ctx
    self.base = base
    self.T = ctx.fp_as_str()
    self.dbl = self.T == 'double'
    self.VEC = 2 if self.dbl else 4
    self.VT = 'double2' if self.dbl else 'float4'
    self.FMA = 'fma' if self.dbl else 'fmaf'
    self.BT = plan.params['threads']
    self.LC = plan.params['chunk']
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

  # ------------------------------------------------------------------ tables
  def _tables(self):
    s = self.s
    self.a_off, self.a_cols = [], []
    off = 0
    gather = []
    for t in s.terms:
      cols = a_values(t)
      self.a_cols.append(cols)
      self.a_off.append(off)
      n = 0
      for _, rows in cols:
        for _, pos in rows:
          gather.append(pos)
          n += 1
      pad = (-n) % self.VEC
      gather.extend([-1] * pad)
      off += n + pad
    self.a_total = off
    self.a_gather = gather
    self.slot_hdr, self.slot_max = [], []
    pairs, hdr = [], []
    for t in s.terms:
      if t.R is None:
        self.slot_hdr.append(-1)
        self.slot_max.append(0)
        continue
      sl = r_slots(t)
      self.slot_hdr.append(len(hdr))
      self.slot_max.append(max(len(c) for c in sl))
      for j in range(s.N):
        hdr.append((len(pairs), len(sl[j])))
        for m, pos in sl[j]:
          pairs.append((m * t.K, pos))
    self.hdr, self.pairs = hdr, pairs
    self.zero_len = max([self.LC] + [self.s.M]) + 4

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

  # ------------------------------------------------------------------ emit
  def emit(self, globals_):
    s = self.s
    T, BT, VT = self.T, self.BT, self.VT
    self._tables()
    b = self.base
    kname = f'kernel_{b}'
    self.w(f'// generated by tensorforge_b200 (strategy: colprog, threads={BT}, chunk={self.LC})')
    self.w('// meta data:')
    for o in self.chain.operands:
      self.w(f'// {o.tensor.gen_descr()}')
    for st in self.chain.stages:
      self.w(f'// {st.descr}')
    g = self.a_gather
    self.w(f'__device__ const int agather_{b}[{max(1, len(g))}] = {{{", ".join(str(x) for x in g) or "0"}}};')
    if self.hdr:
      self.w(f'__device__ const int2 shdr_{b}[{len(self.hdr)}] = {{{", ".join(f"{{{a},{c}}}" for a, c in self.hdr)}}};')
      self.w(f'__device__ const int2 spair_{b}[{max(1, len(self.pairs))}] = {{{", ".join(f"{{{a},{c}}}" for a, c in self.pairs) or "{0,0}"}}};')
    self.w(f'__device__ __align__(16) const {T} zeros_{b}[{self.zero_len}] = {{}};')
    self.w()
    a_bytes = self.a_total * self.ctx.fp_type.size()
    self.smem = (a_bytes + 8 * (len(self.hdr) + len(self.pairs)) + 15) // 16 * 16
    self.w(f'template <bool kVec>')
    mb = self.plan.params.get('min_blocks', 0)
    bounds = f'{BT}, {mb}' if mb else f'{BT}'
    self.w(f'__global__ void __launch_bounds__({bounds}) {kname}({", ".join(self.params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(16) unsigned char tfb_smem_raw[];')
    self.w(f'{T}* const sA = reinterpret_cast<{T}*>(tfb_smem_raw);')
    self.w(f'const {VT}* const sAv = reinterpret_cast<const {VT}*>(tfb_smem_raw);')
    self.w(f'int2* const sHdr = reinterpret_cast<int2*>(tfb_smem_raw + {a_bytes});')
    self.w(f'int2* const sPair = sHdr + {len(self.hdr)};')
    self.open(f'for (int q = threadIdx.x; q < {self.a_total}; q += {BT})')
    self.w(f'const int src = agather_{b}[q];')
    self.w(f'{T} v = {self.lit(0)};')
    for ti, t in enumerate(s.terms):
      lo = self.a_off[ti]
      hi = self.a_off[ti + 1] if ti + 1 < len(s.terms) else self.a_total
      self.w(f'if (q >= {lo} && q < {hi} && src >= 0) v = {t.A.name}[src];')
    self.w('sA[q] = v;')
    self.close()
    if self.hdr:
      self.w(f'for (int q = threadIdx.x; q < {len(self.hdr)}; q += {BT}) sHdr[q] = shdr_{b}[q];')
      self.w(f'for (int q = threadIdx.x; q < {len(self.pairs)}; q += {BT}) sPair[q] = spair_{b}[q];')
    self.w('__syncthreads();')
    self.w(f'const size_t totalCols = numElements * {s.N}u;')
    self.open(f'for (size_t c = (size_t)blockIdx.x * {BT}u + threadIdx.x; c < totalCols; c += (size_t)gridDim.x * {BT}u)')
    self.w(f'const size_t e = c / {s.N}u;')
    self.w(f'const int j = (int)(c - e * {s.N}u);')
    self.w('if (flags != nullptr && flags[e] == 0u) continue;')
    self.w(f'{T} acc[{s.M}];')
    self.w('#pragma unroll')
    self.w(f'for (int i = 0; i < {s.M}; ++i) acc[i] = {self.lit(0)};')
    for ti, t in enumerate(s.terms):
      self._term(ti, t)
    self._store()
    self.close()
    self.ind -= 1
    self.w('}')
    kernel = '\n'.join(self.lines)
    return kernel, self._launch(globals_, kname), ''

  def _launch(self, globals_, kname):
    s = self.s
    BT = self.BT
    args = []
    for t, _ in globals_:
      args.append(t.name)
      if t.addressing.name not in ('NONE', 'SCALAR'):
        args.append(f'{t.name}_extraOffset')
    args += ['numElements', 'flags']
    # 16-byte vector accesses need every strided operand column start aligned
    conds = []
    for o in self.chain.operands:
      if o.kind == 'batched' and o.addressing.name == 'STRIDED':
        conds.append(f'((reinterpret_cast<uintptr_t>({o.name}) & 15u) == 0u)')
        conds.append(f'(({o.name}_extraOffset % {self.VEC}u) == 0u)')
        if o.element_volume() % self.VEC:
          conds.append('false')
    vec_ok = ' && '.join(conds) if conds else 'true'
    kvec = any(o.kind == 'batched' and o.addressing.name == 'STRIDED' for o in self.chain.operands)
    all_cols = all(t.K % self.VEC == 0 for t in s.terms) and s.M % self.VEC == 0
    if not all_cols:
      vec_ok = 'false'
    pre = (f'  const bool useVec = {vec_ok if kvec else "false"};\n'
           f'  static int occ[2][64];\n'
           f'  const int vi = useVec ? 1 : 0;\n'
           f'  if (device < 64 && occ[vi][device] == 0) {{\n'
           f'    int sms = 0, per = 0;\n'
           f'    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);\n'
           f'    if (useVec) {{ cudaFuncSetAttribute({kname}<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, {self.smem});\n'
           f'      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, {kname}<true>, {BT}, {self.smem}); }}\n'
           f'    else {{ cudaFuncSetAttribute({kname}<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, {self.smem});\n'
           f'      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, {kname}<false>, {BT}, {self.smem}); }}\n'
           f'    occ[vi][device] = (per > 0 ? per : 1) * (sms > 0 ? sms : 1);\n'
           f'  }}\n'
           f'  const size_t cap = device < 64 ? (size_t)occ[vi][device] : (size_t)1024;\n'
           f'  if (grid.x > cap) grid.x = (unsigned)cap;\n'
           f'  if (useVec) {kname}<true><<<grid, block, {self.smem}, stream>>>({", ".join(args)});\n'
           f'  else {kname}<false><<<grid, block, {self.smem}, stream>>>({", ".join(args)});\n'
           f'  CHECK_ERR;\n'
           f'  return;')
    self.plan.smem_bytes = self.smem
    return {'kernel': f'{kname}<false>', 'block': BT, 'elements_per_block': 1, 'smem': self.smem,
            'args': args, 'grid': f'(numElements * {s.N}u + {BT} - 1) / {BT}', 'pre': pre}

  # ------------------------------------------------------------------ pieces
  def _base(self, op, var):
    T = self.T
    const = 'const ' if op.is_const else ''
    a = op.addressing.name
    if a == 'STRIDED':
      self.w(f'{const}{T}* const {var} = {op.name} + e * {op.element_volume()}u + {op.name}_extraOffset;')
    elif a == 'PTR_BASED':
      self.w(f'{const}{T}* const {var} = {op.name}[e] + {op.name}_extraOffset;')
    else:
      self.w(f'{const}{T}* const {var} = {op.name};')

  def _vec_ok(self, op):
    return op.addressing.name == 'STRIDED'

  def _accumulate_run(self, ptr, n, dst, scale, vec):
    """dst[0..n) (+)= scale * ptr[0..n)."""
    VEC, VT, FMA = self.VEC, self.VT, self.FMA
    comps = ['x', 'y', 'z', 'w'][:VEC]
    nv = n // VEC if vec else 0
    for v in range(nv):
      self.w(f'{{ const {VT} t = __ldg(reinterpret_cast<const {VT}*>({ptr}) + {v});')
      for ci, cmp in enumerate(comps):
        i = v * VEC + ci
        self.w(f'  {dst}[{i}] = ' + (f't.{cmp};' if scale is None else f'{FMA}({scale}, t.{cmp}, {dst}[{i}]);'))
      self.w('}')
    for i in range(nv * VEC, n):
      self.w(f'{dst}[{i}] = ' + (f'__ldg({ptr} + {i});' if scale is None else f'{FMA}({scale}, __ldg({ptr} + {i}), {dst}[{i}]);'))

  def _term(self, ti, t):
    T, VEC, VT, FMA, LC = self.T, self.VEC, self.VT, self.FMA, self.LC
    s = self.s
    b = self.base
    self.w(f'// term {ti}: A={t.A.name} ({t.A.shape[0]}x{t.A.shape[1]}, {"sparse" if t.A.sparse else "dense"}), '
           f'B={t.B.name}, R={t.R.name if t.R is not None else "-"}')
    self.open('')
    self._base(t.B, 'pB')
    vec = self._vec_ok(t.B)
    ms = self.slot_max[ti]
    if t.R is not None:
      self._base(t.R, 'pR')
      self.w(f'const int2 hdr = sHdr[{self.slot_hdr[ti]} + j];')
      for sl in range(ms):
        self.w(f'const int2 pr{sl} = sPair[hdr.x + ({sl} < hdr.y ? {sl} : 0)];')
        self.w(f'const {T}* const col{sl} = ({sl} < hdr.y) ? pB + pr{sl}.x : zeros_{b};')
        self.w(f'const {T} r{sl} = ({sl} < hdr.y) ? __ldg(pR + pr{sl}.y) : {self.lit(0)};')
    q = self.a_off[ti]
    cols = self.a_cols[ti]
    comps = ['x', 'y', 'z', 'w'][:VEC]
    for l0 in range(0, t.K, LC):
      n = min(LC, t.K - l0)
      self.open('')
      self.w(f'{T} u[{n}];')
      if t.R is None:
        if vec:
          self.open('if (kVec)')
          self._accumulate_run(f'(pB + j * {t.K} + {l0})', n, 'u', None, True)
          self.close()
          self.open('else')
          self._accumulate_run(f'(pB + j * {t.K} + {l0})', n, 'u', None, False)
          self.close()
        else:
          self._accumulate_run(f'(pB + j * {t.K} + {l0})', n, 'u', None, False)
      else:
        self.w('#pragma unroll')
        self.w(f'for (int i = 0; i < {n}; ++i) u[i] = {self.lit(0)};')
        for sl in range(ms):
          # inactive slots point at the zero buffer: they add 0 * 0
          if vec:
            self.open('if (kVec)')
            self._accumulate_run(f'(col{sl} + ({sl} < hdr.y ? {l0} : 0))', n, 'u', f'r{sl}', True)
            self.close()
            self.open('else')
            self._accumulate_run(f'(col{sl} + ({sl} < hdr.y ? {l0} : 0))', n, 'u', f'r{sl}', False)
            self.close()
          else:
            self._accumulate_run(f'(col{sl} + ({sl} < hdr.y ? {l0} : 0))', n, 'u', f'r{sl}', False)
      cur = None
      for l in range(l0, l0 + n):
        for (i, _pos) in cols[l][1]:
          vidx = q // VEC
          if cur != vidx:
            self.w(f'const {VT} a{vidx} = sAv[{vidx}];')
            cur = vidx
          self.w(f'acc[{i}] = {FMA}(a{vidx}.{comps[q % VEC]}, u[{l - l0}], acc[{i}]);')
          q += 1
      self.close()
    self.close()

  def _store(self):
    s = self.s
    T, VEC, VT = self.T, self.VEC, self.VT
    o = s.out
    self._base(o, 'pO')
    self.w(f'{T}* const col = pO + (size_t)j * {s.M};')
    if s.accumulate:
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {s.M}; ++i) acc[i] += col[i];')
    if self._vec_ok(o) and s.M % VEC == 0:
      self.open('if (kVec)')
      for v in range(s.M // VEC):
        vals = ', '.join(f'acc[{v * VEC + c}]' for c in range(VEC))
        self.w(f'reinterpret_cast<{VT}*>(col)[{v}] = make_{VT}({vals});')
      self.close()
      self.open('else')
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {s.M}; ++i) col[i] = acc[i];')
      self.close()
    else:
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {s.M}; ++i) col[i] = acc[i];')
