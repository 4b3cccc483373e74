"""Column-program generator (CUDA cores) for shared-left GEMM chains.

One thread computes one output column (e, j) of out_e = sum_t A_t * B_{e,t} * R_{e,t}:

  1. u = column j of V_t = B_{e,t} * R_{e,t}: the nonzeros (m, r) of column j of R_t are
     walked from a small shared-memory table and u += r * B_{e,t}[:, m] is accumulated
     with 16-byte loads of the contiguous column (in chunks of `chunk` rows).
  2. acc += A_t * u: fully unrolled over A_t's compile-time nonzero pattern, so only
     nonzeros cost an FFMA. A_t's values are staged once per CTA in shared memory in
     exactly the order the FFMAs consume them and read as 128-bit broadcast loads
     (one load feeds 4 FP32 / 2 FP64 FMAs).
  3. out_e[:, j] (+)= acc, stored as one contiguous column.

Intermediates never leave registers; B, R and out are touched once per element, so
HBM traffic is the algorithmic minimum. The grid is persistent (SMs x occupancy) and
walks the flat column space, so any element count and any N is load balanced.
The contraction order differs from the reference's (T_t = A_t*B first, then T_t*R_t);
the result agrees within FP32 rounding (tests hold it to 1e-5 of the output scale).
"""
from .. import plan as _plan
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
    """A-value gather tables and R slot tables (device constants copied to smem)."""
    s = self.s
    self.a_off = []
    self.a_cols = []
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
    # slots: per term with R: start/count per column j, then (m*K, pos) pairs
    self.slot_hdr = []   # per term: offset of its (start,count) table in the int2 array
    pairs = []
    hdr = []
    self.slot_max = []
    for ti, t in enumerate(s.terms):
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
    self.hdr = hdr
    self.pairs = pairs

  # ------------------------------------------------------------------ emit
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

  def emit(self, globals_):
    s = self.s
    T, BT, VEC, VT = self.T, self.BT, self.VEC, self.VT
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
    self.w()
    a_bytes = self.a_total * self.ctx.fp_type.size()
    self.smem = a_bytes + 8 * (len(self.hdr) + len(self.pairs))
    self.smem = (self.smem + 15) // 16 * 16
    self.w(f'__global__ void __launch_bounds__({BT}) {kname}({", ".join(self.params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(16) unsigned char tfb_smem_raw[];')
    self.w(f'{T}* const sA = reinterpret_cast<{T}*>(tfb_smem_raw);')
    self.w(f'const {VT}* const sAv = reinterpret_cast<const {VT}*>(tfb_smem_raw);')
    self.w(f'int2* const sHdr = reinterpret_cast<int2*>(tfb_smem_raw + {a_bytes});')
    self.w(f'int2* const sPair = sHdr + {len(self.hdr)};')
    # stage A values of every term in consumption order
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
      self.open(f'for (int q = threadIdx.x; q < {len(self.hdr)}; q += {BT})')
      self.w(f'sHdr[q] = shdr_{b}[q];')
      self.close()
      self.open(f'for (int q = threadIdx.x; q < {len(self.pairs)}; q += {BT})')
      self.w(f'sPair[q] = spair_{b}[q];')
      self.close()
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
    args = []
    for t, _ in globals_:
      args.append(t.name)
      if t.addressing.name not in ('NONE', 'SCALAR'):
        args.append(f'{t.name}_extraOffset')
    args += ['numElements', 'flags']
    pre = (f'  static int occ[64];\n'
           f'  if (device < 64 && occ[device] == 0) {{\n'
           f'    int sms = 0, per = 0;\n'
           f'    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);\n'
           f'    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, {kname}, {BT}, {self.smem});\n'
           f'    occ[device] = (per > 0 ? per : 1) * (sms > 0 ? sms : 1);\n'
           f'  }}\n'
           f'  const size_t cap = device < 64 ? (size_t)occ[device] : (size_t)1024;\n'
           f'  if (grid.x > cap) grid.x = (unsigned)cap;')
    launch = {'kernel': kname, 'block': BT, 'elements_per_block': 1, 'smem': self.smem, 'args': args,
              'grid': f'(numElements * {s.N}u + {BT} - 1) / {BT}', 'pre': pre}
    self.plan.smem_bytes = self.smem
    return kernel, launch, ''

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

  def _load_run(self, ptr, n, dst, scale=None):
    """dst[0..n) (+)= (scale *) ptr[0..n): 16-byte loads when the address allows it."""
    VEC, VT, FMA = self.VEC, self.VT, self.FMA
    comps = ['x', 'y', 'z', 'w'][:VEC]
    nv = n // VEC
    self.open(f'if ((reinterpret_cast<uintptr_t>({ptr}) & 15u) == 0u)')
    for v in range(nv):
      self.w(f'const {VT} t{v} = __ldg(reinterpret_cast<const {VT}*>({ptr}) + {v});')
      for ci, cmp in enumerate(comps):
        i = v * VEC + ci
        if scale is None:
          self.w(f'{dst}[{i}] = t{v}.{cmp};')
        else:
          self.w(f'{dst}[{i}] = {FMA}({scale}, t{v}.{cmp}, {dst}[{i}]);')
    for i in range(nv * VEC, n):
      if scale is None:
        self.w(f'{dst}[{i}] = __ldg({ptr} + {i});')
      else:
        self.w(f'{dst}[{i}] = {FMA}({scale}, __ldg({ptr} + {i}), {dst}[{i}]);')
    self.close()
    self.open('else')
    self.w('#pragma unroll')
    if scale is None:
      self.w(f'for (int i = 0; i < {n}; ++i) {dst}[i] = __ldg({ptr} + i);')
    else:
      self.w(f'for (int i = 0; i < {n}; ++i) {dst}[i] = {FMA}({scale}, __ldg({ptr} + i), {dst}[i]);')
    self.close()

  def _term(self, ti, t):
    T, VEC, VT, FMA, LC = self.T, self.VEC, self.VT, self.FMA, self.LC
    s = self.s
    self.w(f'// term {ti}: A={t.A.name} ({t.A.shape[0]}x{t.A.shape[1]}, {"sparse" if t.A.sparse else "dense"}), '
           f'B={t.B.name}, R={t.R.name if t.R is not None else "-"}')
    self.open('')
    self._base(t.B, 'pB')
    if t.R is not None:
      self._base(t.R, 'pR')
      self.w(f'const int2 hdr = sHdr[{self.slot_hdr[ti]} + j];')
    q = self.a_off[ti]
    cols = self.a_cols[ti]
    comps = ['x', 'y', 'z', 'w'][:VEC]
    cur_vec = None
    for l0 in range(0, t.K, LC):
      n = min(LC, t.K - l0)
      self.open('')
      self.w(f'{T} u[{n}];')
      if t.R is None:
        self._load_run(f'(pB + j * {t.K} + {l0})', n, 'u')
      else:
        self.w('#pragma unroll')
        self.w(f'for (int i = 0; i < {n}; ++i) u[i] = {self.lit(0)};')
        self.open('for (int sidx = 0; sidx < hdr.y; ++sidx)')
        self.w('const int2 pr = sPair[hdr.x + sidx];')
        self.w(f'const {T} r = pR[pr.y];')
        self.w(f'const {T}* const col = pB + pr.x + {l0};')
        self._load_run('col', n, 'u', scale='r')
        self.close()
      # unrolled sparse FMA block
      cur_vec = None
      for l in range(l0, l0 + n):
        for (i, _pos) in cols[l][1]:
          vidx = q // VEC
          if cur_vec != vidx:
            self.w(f'const {VT} a{vidx} = sAv[{vidx}];')
            cur_vec = vidx
          self.w(f'acc[{i}] = {FMA}(a{vidx}.{comps[q % VEC]}, u[{l - l0}], acc[{i}]);')
          q += 1
      self.close()
    self.close()

  def _store(self):
    s = self.s
    T, VEC, VT = self.T, self.VEC, self.VT
    comps = ['x', 'y', 'z', 'w'][:VEC]
    o = s.out
    self._base(o, 'pO')
    self.w(f'{T}* const col = pO + (size_t)j * {s.M};')
    if s.accumulate:
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {s.M}; ++i) acc[i] += col[i];')
    nv = s.M // VEC
    self.open('if ((reinterpret_cast<uintptr_t>(col) & 15u) == 0u)')
    for v in range(nv):
      vals = ', '.join(f'acc[{v * VEC + c}]' for c in range(VEC))
      self.w(f'reinterpret_cast<{VT}*>(col)[{v}] = make_{VT}({vals});')
    for i in range(nv * VEC, s.M):
      self.w(f'col[{i}] = acc[{i}];')
    self.close()
    self.open('else')
    self.w('#pragma unroll')
    self.w(f'for (int i = 0; i < {s.M}; ++i) col[i] = acc[i];')
    self.close()
