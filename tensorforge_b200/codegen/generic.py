"""Generic sm_100a code generator: any lowered chain, CUDA cores.

Each batch element is owned by a group of `G` lanes; a CTA holds `E` groups. For every
stage the lanes split the destination entries (d = lane, lane+G, ...) and each entry
accumulates its full contraction over the contracted index box, contracted index k0
fastest as in the reference's linearized loop (multilinear.py:105-157). Sparse operands
are expanded once into dense shared-memory boxes (shared ones once per CTA, batched
ones once per element), temporaries live in per-element shared memory (regions whose
live ranges are disjoint share memory: `live_ranges`, `assign_offsets`), and the
destination is updated in global memory stage by stage, exactly in descriptor order.
The grid loops over element tiles, so the same kernel also runs persistently.
"""
from functools import reduce

from ..common.basic_types import FloatingPointType
from ..common.exceptions import GenerationError
from .elementwise import emit_elementwise_stage


def _prod(xs):
  return reduce(lambda a, b: a * b, xs, 1)


def _colmajor(sizes):
  out, acc = [], 1
  for s in sizes:
    out.append(acc)
    acc *= s
  return out


def _sparse_box(op):
  """Dense box used to expand a compactly stored operand: relative to bbox.lower over the pattern's shape."""
  shape = list(op.tensor.spp.indexmask.shape) if hasattr(op.tensor.spp, 'indexmask') else list(op.tensor.shape)
  return shape


def _stage_access(st):
  """(operands written, operands read) by one stage, as sets of operand ids."""
  if getattr(st, 'kind', '') == 'elementwise':
    return {id(o) for o in st.written}, {id(o) for o in st.read}
  reads = {id(r.op) for r in st.ops}
  if st.add:
    reads.add(id(st.dest))
  return {id(st.dest)}, reads


def live_ranges(chain):
  """Live interval [first, last] (stage indices) of every per-element shared-memory region:
  batched sparse operands (expanded right before the first stage reading them, live until
  the last one) and temporaries (from the first stage writing them to the last stage
  touching them). Restates the reference's liveness analysis (backend/opt/liveness.py:
  12-57) over this IR's stages."""
  access = [_stage_access(st) for st in chain.stages]
  out = {}
  for o in chain.operands:
    if o.kind == 'batched' and o.sparse:
      used = [i for i, (_, r) in enumerate(access) if id(o) in r]
      out[o.name] = (min(used), max(used)) if used else (0, 0)
  for t in chain.tmps:
    touched = [i for i, (w, r) in enumerate(access) if id(t) in w or id(t) in r]
    written = [i for i, (w, _) in enumerate(access) if id(t) in w]
    first = min(written) if written else (min(touched) if touched else 0)
    out[t.name] = (first, max(touched) if touched else first)
  return out


def region_sizes(chain):
  """Values per element of every per-element region (expanded sparse box or temporary),
  each rounded up to a multiple of 4 so that every region stays 16-byte aligned."""
  sizes = {}
  for o in chain.operands:
    if o.kind == 'batched' and o.sparse:
      sizes[o.name] = _align4(_prod(_sparse_box(o)))
  for t in chain.tmps:
    sizes[t.name] = _align4(max([s.defines_volume(t) for s in chain.stages] + [0]))
  return sizes


def assign_offsets(sizes, ranges):
  """Offsets (values) for regions whose live intervals may share memory: two regions
  overlap in memory only if their intervals are disjoint. First fit in order of interval
  start (largest first on ties) over an interval graph - the reference's region allocation
  (backend/opt/mem_region_allocation.py:29-94, coloring/coloring.py:24-96) colours the
  same interference relation and sizes each colour by its largest member; first fit by
  offset packs regions of different sizes tighter. Returns ({name: offset}, total)."""
  placed = []
  offsets = {}
  for name in sorted(sizes, key=lambda n: (ranges[n][0], -sizes[n], n)):
    lo, hi = ranges[name]
    busy = sorted((offsets[p], offsets[p] + sizes[p]) for p in placed
                  if not (ranges[p][1] < lo or hi < ranges[p][0]))
    off = 0
    for a, b in busy:
      if off + sizes[name] <= a:
        break
      off = max(off, b)
    offsets[name] = off
    placed.append(name)
  total = max([offsets[n] + sizes[n] for n in sizes] + [0])
  return offsets, _align4(total)


def shared_regions(chain):
  """CTA-shared regions (expanded shared sparse operands): ({name: offset}, total values,
  {names expanded once per CTA}). Operands whose memory no other region uses are expanded
  once per CTA; when the resident layout would not fit next to the per-element regions,
  operands with disjoint live ranges share memory and are expanded again, per tile, right
  before the first stage reading them."""
  ops = [o for o in chain.operands if o.kind == 'shared' and o.sparse]
  sizes = {o.name: _align4(_prod(_sparse_box(o))) for o in ops}
  resident_total = sum(sizes.values())
  offsets, off = {}, 0
  for o in ops:
    offsets[o.name] = off
    off += sizes[o.name]
  _, per_elem = assign_offsets(region_sizes(chain), live_ranges(chain))
  if (resident_total + per_elem) * chain.fp.size() <= 227 * 1024 or len(ops) < 2:
    return offsets, resident_total, {o.name for o in ops}
  access = [_stage_access(st) for st in chain.stages]
  ranges = {}
  for o in ops:
    used = [i for i, (_, r) in enumerate(access) if id(o) in r]
    ranges[o.name] = (min(used), max(used)) if used else (0, 0)
  offsets, total = assign_offsets(sizes, ranges)
  resident = set()
  for n in sizes:
    lo, hi = offsets[n], offsets[n] + sizes[n]
    if not any(m != n and offsets[m] < hi and lo < offsets[m] + sizes[m] for m in sizes):
      resident.add(n)
  return offsets, total, resident


def smem_layout(chain):
  """(values in the CTA-shared region, values per element) for the generic generator,
  with regions reusing memory across disjoint live ranges."""
  _, shared, _ = shared_regions(chain)
  _, per_elem = assign_offsets(region_sizes(chain), live_ranges(chain))
  return shared, per_elem


def _align4(x):
  return (x + 3) // 4 * 4


class GenericEmitter:
  def __init__(self, chain, plan, context, base_name):
    self.chain = chain
    self.plan = plan
    self.ctx = context
    self.base = base_name
    self.T = context.fp_as_str()
    self.G = plan.params['threads_per_element']
    self.E = plan.params['elements_per_block']
    self.lines = []
    self.ind = 0

  # ---------------------------------------------------------------- writer
  def w(self, s=''):
    self.lines.append('  ' * self.ind + s)

  def block(self, head):
    emitter = self

    class _B:
      def __enter__(self_):
        emitter.w(head + ' {')
        emitter.ind += 1

      def __exit__(self_, *a):
        emitter.ind -= 1
        emitter.w('}')
    return _B()

  def lit(self, v):
    return self.ctx.fp_type.literal(v)

  # ---------------------------------------------------------------- layout
  def _regions(self):
    regions = {}
    soff, shared, self.resident = shared_regions(self.chain)
    for o in self.chain.operands:
      if o.kind == 'shared' and o.sparse:
        regions[o.name] = ('shared', soff[o.name], _sparse_box(o))
    offsets, per_elem = assign_offsets(region_sizes(self.chain), live_ranges(self.chain))
    for o in self.chain.operands:
      if o.kind == 'batched' and o.sparse:
        regions[o.name] = ('elem', offsets[o.name], _sparse_box(o))
    for t in self.chain.tmps:
      regions[t.name] = ('elem', offsets[t.name], None)
    return regions, shared, per_elem

  # ---------------------------------------------------------------- access
  def _value(self, ref, idx_exprs, regions):
    o = ref.op
    if o.kind == 'scalar':
      return o.name
    if o.kind == 'data':
      return self._data_value(o, ref, idx_exprs)
    if o.kind == 'tmp':
      terms = [f'({e} - {org}) * {st}' for e, org, st in zip(idx_exprs, ref.origin, ref.strides)]
      return f'tmp_{o.name}[{" + ".join(terms) or "0"}]'
    if o.sparse:
      box = _sparse_box(o)
      strides = _colmajor(box)
      lower = o.bbox.lower()
      terms = [f'({e} - {lo}) * {st}' for e, lo, st in zip(idx_exprs, lower, strides)]
      return f'dn_{o.name}[{" + ".join(terms) or "0"}]'
    terms = [f'({e} - {org}) * {st}' for e, org, st in zip(idx_exprs, ref.origin, ref.strides)]
    return f'glb_{o.name}[{" + ".join(terms) or "0"}]'

  def _data_value(self, o, ref, idx_exprs):
    data = o.tensor.data
    if len(ref.target) == 0:
      if isinstance(data, dict):
        return self.lit(data.get((), 0.0))
      return self.lit(float(data[0]))
    # small compile-time table, dense over the operand shape
    return f'data_{o.name}[{" + ".join(f"({e}) * {st}" for e, st in zip(idx_exprs, _colmajor(list(o.shape))))}]'

  # ---------------------------------------------------------------- emit
  def kernel_params(self, globals_):
    params = []
    for t, _ in globals_:
      dt = self.T if t.datatype is None else str(t.datatype)
      if t.addressing.name == 'SCALAR':
        params.append(f'{dt} {t.name}')
      else:
        const = 'const ' if t.direction.name == 'SOURCE' else ''
        params.append(f'{const}{dt}{t.addressing.to_pointer()} {t.name}')
        if t.addressing.name != 'NONE':
          params.append(f'unsigned {t.name}_extraOffset')
    params += ['size_t numElements', 'const unsigned* flags']
    return params

  def emit_kernel(self, globals_):
    chain = self.chain
    T, G, E = self.T, self.G, self.E
    regions, shared_vals, per_elem = self._regions()
    kname = f'kernel_{self.base}'
    self.w(f'// generated by tensorforge_b200 (strategy: generic, G={G}, E={E})')
    for line in self._meta():
      self.w(line)
    # compile-time tables
    for o in chain.operands:
      if o.kind == 'data' and len(o.shape) > 0:
        vals = [0.0] * max(1, _prod(o.shape))
        if isinstance(o.tensor.data, dict):
          for idx, v in o.tensor.data.items():
            pos = sum(i * s for i, s in zip(idx, _colmajor(list(o.shape))))
            vals[pos] = v
        self.w(f'__device__ const {T} data_{o.name}_{self.base}[{len(vals)}] = {{{", ".join(self.lit(v) for v in vals)}}};')
      if o.sparse:
        box = _sparse_box(o)
        strides = _colmajor(box)
        lower = o.bbox.lower()
        pairs = []
        for idx, pos in o.nonzeros():
          rel = [i - lo for i, lo in zip(idx, lower)]
          pairs.append((pos, sum(r * s for r, s in zip(rel, strides))))
        pairs.sort()
        self.w(f'__device__ const unsigned short scat_{o.name}_{self.base}[{max(1, len(pairs))}] = '
               f'{{{", ".join(str(d) for _, d in pairs) or "0"}}};')
        self.w(f'__device__ const unsigned short spos_{o.name}_{self.base}[{max(1, len(pairs))}] = '
               f'{{{", ".join(str(p) for p, _ in pairs) or "0"}}};')
    self.w()
    self.w(f'__global__ void __launch_bounds__({G * E}) {kname}({", ".join(self.kernel_params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(16) unsigned char tfb_smem_raw[];')
    self.w(f'{T}* const tfb_smem = reinterpret_cast<{T}*>(tfb_smem_raw);')
    for o in chain.operands:
      if o.kind == 'data' and len(o.shape) > 0:
        self.w(f'const {T}* const data_{o.name} = data_{o.name}_{self.base};')
    # shared sparse operands: resident ones expanded once per CTA, the others (sharing
    # memory with another shared region) per tile before their first stage
    for o in chain.operands:
      if o.kind == 'shared' and o.sparse:
        _, off, box = regions[o.name]
        self.w(f'{T}* const dn_{o.name} = tfb_smem + {off};')
        if o.name in self.resident:
          self._expand_shared(o, box)
    self.w('__syncthreads();')
    self.w(f'const unsigned slot = threadIdx.x / {G}u;')
    self.w(f'const unsigned lane = threadIdx.x % {G}u;')
    self.w(f'{T}* const elem_smem = tfb_smem + {shared_vals} + slot * {per_elem}u;')
    for name, (where, off, box) in regions.items():
      if where == 'elem':
        pref = 'dn_' if box is not None else 'tmp_'
        self.w(f'{T}* const {pref}{name} = elem_smem + {off};')
    sync = '__syncwarp()' if G <= 32 else '__syncthreads()'
    with self.block(f'for (size_t tile = blockIdx.x; tile * {E}u < numElements; tile += gridDim.x)'):
      self.w(f'const size_t batchId = tile * {E}u + slot;')
      self.w('bool active = batchId < numElements;')
      self.w('if (active && flags != nullptr) active = flags[batchId] != 0u;')
      # element base pointers
      for o in chain.operands:
        if o.kind not in ('batched', 'shared'):
          continue
        const = 'const ' if o.is_const else ''
        a = o.addressing.name
        if a == 'NONE':
          self.w(f'{const}{T}* const glb_{o.name} = {o.name};')
        elif a == 'STRIDED':
          self.w(f'{const}{T}* const glb_{o.name} = active ? {o.name} + batchId * {o.element_volume()}u + {o.name}_extraOffset : nullptr;')
        else:
          self.w(f'{const}{T}* const glb_{o.name} = active ? {o.name}[batchId] + {o.name}_extraOffset : nullptr;')
      first_use = live_ranges(chain)
      access = [_stage_access(st) for st in chain.stages]
      shared_first = {}
      for o in chain.operands:
        if o.kind == 'shared' and o.sparse:
          used = [i for i, (_, r) in enumerate(access) if id(o) in r]
          shared_first[o.name] = min(used) if used else 0
      for si, st in enumerate(chain.stages):
        # batched sparse operands are expanded right before the first stage that reads them
        # (their region may reuse the memory of regions that are dead by then)
        shared_now = [o for o in chain.operands if o.kind == 'shared' and o.sparse and o.name not in self.resident
                      and shared_first[o.name] == si]
        if shared_now:
          self.w('__syncthreads();  // every element group is done with the region\'s previous operand')
          for o in shared_now:
            self._expand_shared(o, regions[o.name][2])
          self.w('__syncthreads();')
        expand = [o for o in chain.operands if o.kind == 'batched' and o.sparse and first_use[o.name][0] == si]
        if expand:
          for o in expand:
            _, off, box = regions[o.name]
            with self.block(f'for (unsigned i = lane; i < {_prod(box)}u; i += {G}u)'):
              self.w(f'dn_{o.name}[i] = {self.lit(0)};')
          self.w(f'{sync};')
          for o in expand:
            nnz = len(o.nonzeros())
            with self.block(f'if (active) for (unsigned i = lane; i < {nnz}u; i += {G}u)'):
              self.w(f'dn_{o.name}[scat_{o.name}_{self.base}[i]] = glb_{o.name}[spos_{o.name}_{self.base}[i]];')
          self.w(f'{sync};')
        self.w(f'// stage {si}: {st.descr}'.replace('\n', ' '))
        with self.block('if (active)'):
          if getattr(st, 'kind', '') == 'elementwise':
            emit_elementwise_stage(self, st)
          else:
            self._emit_stage(st, regions)
        self.w(f'{sync};')
    self.ind -= 1
    self.w('}')
    return '\n'.join(self.lines)

  def _expand_shared(self, o, box):
    """Zero the dense box of shared sparse operand `o` and scatter its nonzeros (all CTA threads)."""
    vol = _prod(box)
    nnz = len(o.nonzeros())
    with self.block(f'for (unsigned i = threadIdx.x; i < {vol}u; i += blockDim.x)'):
      self.w(f'dn_{o.name}[i] = {self.lit(0)};')
    self.w('__syncthreads();')
    with self.block(f'for (unsigned i = threadIdx.x; i < {nnz}u; i += blockDim.x)'):
      self.w(f'dn_{o.name}[scat_{o.name}_{self.base}[i]] = {o.name}[spos_{o.name}_{self.base}[i]];')

  def _meta(self):
    out = ['// meta data:']
    for o in self.chain.operands:
      out.append(f'// {o.tensor.gen_descr()}')
    for st in self.chain.stages:
      out.append(f'// {st.descr}')
    return out

  def _emit_stage(self, st, regions):
    T, G = self.T, self.G
    sizes = [u - l for l, u in st.n_ranges]
    vol = _prod(sizes)
    with self.block(f'for (unsigned d = lane; d < {vol}u; d += {G}u)'):
      rem = 'd'
      for i, ((lo, up), s) in enumerate(zip(st.n_ranges, sizes)):
        div = _prod(sizes[:i])
        expr = f'(d / {div}u) % {s}u' if div > 1 else f'd % {s}u'
        self.w(f'const int n{i} = {lo} + (int)({expr});')
      self.w(f'{T} acc = {self.lit(0)};')
      # loops over contracted indices, k0 innermost
      nk = len(st.k_ranges)
      for i in reversed(range(nk)):
        lo, up = st.k_ranges[i]
        self.w('#pragma unroll 4')
        self.w(f'for (int k{i} = {lo}; k{i} < {up}; ++k{i}) {{')
        self.ind += 1
      vals = []
      for ref in st.ops:
        idx = [f'n{t}' if t >= 0 else f'k{-t - 1}' for t in ref.target]
        vals.append(self._value(ref, idx, regions))
      prod = ' * '.join(vals) if vals else self.lit(0)
      self.w(f'acc += {prod};')
      for i in range(nk):
        self.ind -= 1
        self.w('}')
      idx = [f'n{i}' for i in range(len(st.n_ranges))]
      terms = [f'({e} - {org}) * {s}' for e, org, s in zip(idx, st.dest_origin, st.dest_strides)]
      addr = ' + '.join(terms) or '0'
      target = f'tmp_{st.dest.name}[{addr}]' if st.dest.kind == 'tmp' else f'glb_{st.dest.name}[{addr}]'
      if st.add:
        self.w(f'{target} = acc + {target};')
      else:
        self.w(f'{target} = acc;')


def emit_generic(chain, plan, context, base_name, globals_):
  em = GenericEmitter(chain, plan, context, base_name)
  kernel = em.emit_kernel(globals_)
  args = []
  for t, _ in globals_:
    args.append(t.name)
    if t.addressing.name not in ('NONE', 'SCALAR'):
      args.append(f'{t.name}_extraOffset')
  args += ['numElements', 'flags']
  launch = {
    'kernel': f'kernel_{base_name}',
    'block': plan.params['threads_per_element'] * plan.params['elements_per_block'],
    'elements_per_block': plan.params['elements_per_block'],
    'smem': plan.smem_bytes,
    'args': args,
  }
  return kernel, launch
