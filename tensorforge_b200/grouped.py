"""Mixed-shape batched launches: one persistent kernel over a device work table.

A `GroupedKernel` fuses several generated chains of the shared-left form (plan/chains.py),
typically the same operation at different basis sizes and quantity counts, into one
persistent kernel:

  * each group contributes a tile function (codegen/colprog.py, CUDA cores, A staged in
    shared memory) specialised at generation time for its shape and sparsity patterns;
  * a device work table lists (group, tile) items ordered by group; CTAs (SMs x
    occupancy) pull items with one atomic counter and run the matching tile function,
    restaging the group's A values only when their group changes;
  * the counter is reset on the launch stream, so launch + reset can be captured in a CUDA
    graph and replayed (`capture()`).

C ABI of the emitted library (one per fused set):

    int tfb_grouped_launch_<name>(const tfb_group_args* args, const uint2* items,
                                  unsigned num_items, unsigned* counter, void* stream);

`args[g]` holds group g's ABI symbols in its launcher order (pointer or pointer array,
extra offset), its element count and flags; `items` are (group, tile) pairs; `counter` is
one device word of scratch that the launcher zeroes before the kernel.
"""
import ctypes
import hashlib

from .common.basic_types import Addressing
from .common.exceptions import GenerationError
from .plan import Plan
from .plan.chains import match_left_chain
from .codegen.colprog import _ColProg, _pad
from .runtime.build import build_library

MAX_SYMBOLS = 16

ARGS_STRUCT = '''
#include "tensorforge_b200_grouped.h"
'''


class _GroupArgs(ctypes.Structure):
  _fields_ = [('ptr', ctypes.c_void_p * MAX_SYMBOLS), ('off', ctypes.c_uint * MAX_SYMBOLS),
              ('num_elements', ctypes.c_ulonglong), ('flags', ctypes.c_void_p)]


class GroupedKernel:
  def __init__(self, generators, threads=256, name=None, prefetch=True):
    if not generators:
      raise GenerationError('a grouped launch needs at least one chain')
    self.gens = generators
    self.threads = threads
    fp = {g.get_context().fp_type for g in generators}
    if len(fp) != 1:
      raise GenerationError('all groups of a grouped launch must use the same precision')
    self.T = generators[0].get_context().fp_as_str()
    self.fs = 8 if self.T == 'double' else 4
    for g in generators:
      if g.get_chain() is None:
        g.generate()
      shape = match_left_chain(g.get_chain())
      if shape is None or shape.epilogue:
        raise GenerationError(f'{g.get_base_name()} is not a shared-left chain without elementwise stages')
      for t, stype in g.abi_symbols():
        if t.addressing == Addressing.SCALAR:
          raise GenerationError('scalar operands are not supported in grouped launches')
      if len(g.abi_symbols()) > MAX_SYMBOLS:
        raise GenerationError(f'at most {MAX_SYMBOLS} operands per group')
    # prefetch: each group's tile fetches the next work item's inputs (same group) into a
    # cp.async stage during its last K stage, as the standalone column programs do (config 3,
    # 1.5M mixed-shape elements: 33.9 ms against 38.5 ms without; 128 threads per CTA
    # measured 40.3 ms without and 59.5 ms with the stage, whose shared memory then leaves
    # one CTA per SM)
    self.prefetch = bool(prefetch)
    key = ','.join(g.get_base_name() for g in generators) + f'|{threads}' + ('|pf' if self.prefetch else '')
    self.name = name or 'grouped_' + hashlib.md5(key.encode()).hexdigest()[:10]
    self._emit()
    self._lib = None

  def _emit(self):
    parts, work_vals, a_vals, self.tiles_per = [], 0, 0, []
    self.te = []
    for gid, g in enumerate(self.gens):
      shape = match_left_chain(g.get_chain())
      plan = Plan('colprog', {'threads': self.threads, 'chunk': 16, 'a_source': 'smem',
                              'prefetch': 1 if self.prefetch else 0})
      em = _ColProg(g.get_chain(), shape, plan, g.get_context(), f'{self.name}_g{gid}')
      parts.append(em.emit_group_functions(g.abi_symbols(), gid))
      work_vals = max(work_vals, em.work_vals + em.stage_vals)
      a_vals = max(a_vals, _pad(em.a_total, 4))
      self.te.append(em.TE)
    self.smem = (work_vals + a_vals) * self.fs
    if self.smem > 227 * 1024:
      raise GenerationError(f'grouped launch needs {self.smem} bytes of shared memory')
    T, BT = self.T, self.threads
    k = []
    k.append(f'__global__ void __launch_bounds__({BT}) kernel_{self.name}(const tfb_group_args* __restrict__ args, '
             'const uint2* __restrict__ items, unsigned num_items, unsigned* __restrict__ counter) {')
    k.append('  extern __shared__ __align__(16) unsigned char tfb_smem_raw[];')
    k.append(f'  {T}* const ubuf = reinterpret_cast<{T}*>(tfb_smem_raw);')
    k.append(f'  {T}* const sA = ubuf + {work_vals};')
    k.append('  // the next item is claimed while the current one runs (the atomic\'s latency is hidden)')
    k.append('  __shared__ unsigned s_item[2];')
    k.append('  if (threadIdx.x == 0) s_item[0] = atomicAdd(counter, 1u);')
    k.append('  __syncthreads();')
    k.append('  unsigned item = s_item[0], nb = 1u;')
    k.append('  int cur = -1;')
    k.append('  for (;;) {')
    k.append('    if (item >= num_items) break;')
    k.append('    if (threadIdx.x == 0) s_item[nb] = atomicAdd(counter, 1u);')
    k.append('    const uint2 wi = items[item];')
    k.append('    if ((int)wi.x != cur) {')
    k.append('      switch (wi.x) {')
    for gid in range(len(self.gens)):
      pf = f' group{gid}_prefetch(args[{gid}], (size_t)wi.y, ubuf);' if self.prefetch else ''
      k.append(f'        case {gid}u: group{gid}_stage_a(args[{gid}], sA);{pf} break;')
    k.append('        default: break;')
    k.append('      }')
    if self.prefetch:
      k.append('      tfb_cp::commit();')
    k.append('      __syncthreads();')
    k.append('      cur = (int)wi.x;')
    k.append('    }')
    nxt = ''
    if self.prefetch:
      # the claimed next item, known to every thread, decides the prefetch of this tile
      k.append('    __syncthreads();')
      k.append('    const unsigned nx = s_item[nb];')
      k.append('    size_t next_tile = ~(size_t)0;')
      k.append('    if (nx < num_items) { const uint2 wn = items[nx]; if (wn.x == wi.x) next_tile = (size_t)wn.y; }')
      nxt = ', next_tile'
    k.append('    switch (wi.x) {')
    for gid in range(len(self.gens)):
      k.append(f'      case {gid}u: group{gid}_tile(args[{gid}], (size_t)wi.y, ubuf, sA{nxt}); break;')
    k.append('      default: break;')
    k.append('    }')
    k.append('    __syncthreads();')
    k.append('    item = s_item[nb];')
    k.append('    nb ^= 1u;')
    k.append('  }')
    if self.prefetch:
      k.append('  tfb_cp::wait_all();')
    k.append('}')
    k.append('')
    k.append(f'extern "C" int tfb_grouped_launch_{self.name}(const void* args, const void* items, unsigned num_items, '
             'unsigned* counter, void* streamPtr) {')
    k.append('  cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);')
    k.append('  if (num_items == 0) return 0;')
    k.append('  int device = 0, sms = 0, per = 0;')
    k.append('  cudaGetDevice(&device);')
    k.append('  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);')
    k.append(f'  cudaFuncSetAttribute(kernel_{self.name}, cudaFuncAttributeMaxDynamicSharedMemorySize, {self.smem});')
    k.append(f'  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel_{self.name}, {BT}, {self.smem});')
    k.append('  unsigned grid = (unsigned)((per > 0 ? per : 1) * (sms > 0 ? sms : 1));')
    k.append('  if (grid > num_items) grid = num_items;')
    k.append('  cudaMemsetAsync(counter, 0, sizeof(unsigned), stream);')
    k.append(f'  kernel_{self.name}<<<grid, {BT}, {self.smem}, stream>>>(static_cast<const tfb_group_args*>(args), '
             'static_cast<const uint2*>(items), num_items, counter);')
    k.append('  return (int)cudaGetLastError();')
    k.append('}')
    k += self._noalloc_variant(work_vals)
    from .codegen import PRELUDE
    self.source_text = PRELUDE + ARGS_STRUCT + '\n\n'.join(parts) + '\n\n' + '\n'.join(k) + '\n'

  def _noalloc_variant(self, work_vals):
    """An entry point for callers that cannot allocate device memory.

    Some callers cannot call cudaMalloc: code running under an external memory manager
    that owns every device allocation (a host application that hands this library
    pre-sized buffers only), or a latency-critical loop where an allocation could block
    on a device-wide synchronisation. The regular entry point needs two device buffers
    besides the operands (the work table and the work counter); this variant needs
    neither. The group records and per-group tile offsets travel by value as one kernel
    parameter (`__grid_constant__`, so no host buffer is referenced once the call
    returns), and the one piece of device scratch, the work counter, sits in a file-scope
    device array of the library. The caller still passes every input and output.
    """
    T, BT, G = self.T, self.threads, len(self.gens)
    te = ', '.join(str(t) for t in self.te)
    n = self.name
    k = ['',
         '// Scratch of the allocation-free entry point: the work counter that CTAs pull',
         '// tiles from (one word used of TFB_NOALLOC_SCRATCH_WORDS). Every GPU that loads this',
         '// library keeps one copy until the process exits. All calls share it and it keeps',
         '// the last call\'s value; each call clears it on its stream before the kernel, so',
         '// calls ordered on the GPU are independent, and calls that overlap on the GPU',
         '// (different streams, no ordering between them) race on it.',
         f'static __device__ __align__(256) unsigned tfb_noalloc_scratch_{n}[TFB_NOALLOC_SCRATCH_WORDS];',
         '',
         f'struct tfb_noalloc_params_{n} {{',
         '  unsigned num_groups;',
         f'  unsigned tile_prefix[{G + 1}];',
         f'  tfb_group_args args[{G}];',
         '};',
         '',
         f'__global__ void __launch_bounds__({BT}) kernel_{n}_noalloc(const __grid_constant__ tfb_noalloc_params_{n} prm, '
         'unsigned* __restrict__ counter) {',
         '  extern __shared__ __align__(16) unsigned char tfb_smem_raw[];',
         f'  {T}* const ubuf = reinterpret_cast<{T}*>(tfb_smem_raw);',
         f'  {T}* const sA = ubuf + {work_vals};',
         '  __shared__ unsigned s_item, s_group, s_tile;',
         '  const unsigned ngroups = prm.num_groups;',
         '  const unsigned total = prm.tile_prefix[ngroups];',
         '  int cur = -1;',
         '  for (;;) {',
         '    if (threadIdx.x == 0) {',
         '      const unsigned item = atomicAdd(counter, 1u);',
         '      unsigned g = 0;',
         '      while (g + 1u < ngroups && prm.tile_prefix[g + 1u] <= item) ++g;',
         '      s_item = item; s_group = g; s_tile = item - prm.tile_prefix[g];',
         '    }',
         '    __syncthreads();',
         '    const unsigned item = s_item, grp = s_group, tile = s_tile;',
         '    __syncthreads();',
         '    if (item >= total) break;',
         '    if ((int)grp != cur) {',
         '      switch (grp) {']
    for gid in range(G):
      k.append(f'        case {gid}u: group{gid}_stage_a(prm.args[{gid}], sA); break;')
    k += ['        default: break;',
          '      }',
          '      __syncthreads();',
          '      cur = (int)grp;',
          '    }',
          '    switch (grp) {']
    for gid in range(G):
      if self.prefetch:
        # no look-ahead here: the tile's inputs are fetched right before it
        k.append(f'      case {gid}u: group{gid}_prefetch(prm.args[{gid}], (size_t)tile, ubuf); tfb_cp::commit(); '
                 f'group{gid}_tile(prm.args[{gid}], (size_t)tile, ubuf, sA, ~(size_t)0); break;')
      else:
        k.append(f'      case {gid}u: group{gid}_tile(prm.args[{gid}], (size_t)tile, ubuf, sA); break;')
    k += ['      default: break;',
          '    }',
          '    __syncthreads();',
          '  }',
          '}',
          '',
          '// Allocation-free form of tfb_grouped_launch_<set> (declared in',
          '// tensorforge_b200_grouped.h): `host_args` holds num_groups tfb_group_args records in',
          '// host memory, in group order; they are passed to the kernel by value, so the caller may',
          '// reuse that memory as soon as the call returns. Allocates nothing. The first call on a',
          '// device (the current device) looks up the scratch address there with',
          '// cudaGetSymbolAddress and keeps it for the process; make that first call before any',
          '// stream capture. The cached address does not survive cudaDeviceReset. Returns a',
          '// cudaError_t value: cudaErrorInvalidValue for a null `host_args` or for more groups',
          '// than the fused set or TFB_NOALLOC_MAX_GROUPS.',
          f'extern "C" int tfb_grouped_launch_noalloc_{n}(const void* host_args, unsigned num_groups, void* streamPtr) {{',
          f'  static const unsigned tiles_per_group[{G}] = {{{te}}};',
          '  static void* scratch_ptr[64];',
          '  static std::mutex setup_mu;',
          '  cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);',
          '  if (host_args == nullptr) {',
          f'    std::fprintf(stderr, "tfb_grouped_launch_noalloc_{n}: host_args is null\\n");',
          '    return (int)cudaErrorInvalidValue;',
          '  }',
          f'  if (num_groups > {G}u || num_groups > TFB_NOALLOC_MAX_GROUPS) {{',
          f'    std::fprintf(stderr, "tfb_grouped_launch_noalloc_{n}: %u groups requested, at most {min(G, 64)} supported\\n", num_groups);',
          '    return (int)cudaErrorInvalidValue;',
          '  }',
          '  if (num_groups == 0) return 0;',
          '  int device = 0;',
          '  cudaError_t err = cudaGetDevice(&device);',
          '  if (err != cudaSuccess) return (int)err;',
          '  if (device < 0 || device >= 64) return (int)cudaErrorInvalidDevice;',
          '  {',
          '    std::lock_guard<std::mutex> guard(setup_mu);',
          '    if (scratch_ptr[device] == nullptr) {',
          '      void* p = nullptr;',
          f'      err = cudaGetSymbolAddress(&p, tfb_noalloc_scratch_{n});',
          '      if (err != cudaSuccess) return (int)err;',
          '      scratch_ptr[device] = p;',
          '    }',
          '  }',
          f'  tfb_noalloc_params_{n} prm{{}};',
          '  prm.num_groups = num_groups;',
          '  const tfb_group_args* ga = static_cast<const tfb_group_args*>(host_args);',
          '  unsigned long long total = 0;',
          '  for (unsigned g = 0; g < num_groups; ++g) {',
          '    prm.args[g] = ga[g];',
          '    prm.tile_prefix[g] = (unsigned)total;',
          '    total += (ga[g].num_elements + tiles_per_group[g] - 1) / tiles_per_group[g];',
          '    if (total > 0xFFFFFFF0ull) return (int)cudaErrorInvalidValue;',
          '  }',
          '  prm.tile_prefix[num_groups] = (unsigned)total;',
          '  if (total == 0) return 0;',
          '  unsigned* counter = static_cast<unsigned*>(scratch_ptr[device]);',
          '  err = cudaMemsetAsync(counter, 0, sizeof(unsigned), stream);',
          '  if (err != cudaSuccess) return (int)err;',
          '  int sms = 0, per = 0;',
          '  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);',
          f'  cudaFuncSetAttribute(kernel_{n}_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, {self.smem});',
          f'  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel_{n}_noalloc, {BT}, {self.smem});',
          '  unsigned grid = (unsigned)((per > 0 ? per : 1) * (sms > 0 ? sms : 1));',
          '  if (grid > total) grid = (unsigned)total;',
          f'  kernel_{n}_noalloc<<<grid, {BT}, {self.smem}, stream>>>(prm, counter);',
          '  return (int)cudaGetLastError();',
          '}']
    return k

  def source(self):
    return self.source_text

  def build(self):
    self.so_path = build_library(self.source_text)
    return self.so_path

  def _load(self):
    if self._lib is None:
      self.build()
      self._lib = ctypes.CDLL(self.so_path, mode=ctypes.RTLD_LOCAL)
      self._fn = getattr(self._lib, f'tfb_grouped_launch_{self.name}')
      self._fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p]
      self._fn.restype = ctypes.c_int
    return self._fn

  def work_items(self, counts):
    """(group, tile) pairs for element counts per group, ordered by group."""
    items = []
    for gid, n in enumerate(counts):
      tiles = (int(n) + self.te[gid] - 1) // self.te[gid]
      items.extend((gid, t) for t in range(tiles))
    return items

  def prepare(self, group_kwargs):
    """Device argument records, work table and counter for one set of group buffers.

    group_kwargs[g] maps group g's ABI names (as for CompiledKernel calls) to tensors /
    addresses, plus numElements and optional flags. Returns a `GroupedLaunch`.
    """
    import torch
    if len(group_kwargs) != len(self.gens):
      raise ValueError('one argument set per group is required')
    recs = (_GroupArgs * len(self.gens))()
    keep = []
    counts = []
    for gid, (g, kw) in enumerate(zip(self.gens, group_kwargs)):
      rec = recs[gid]
      for i, (t, _) in enumerate(g.abi_symbols()):
        v = kw[t.name]
        rec.ptr[i] = v if isinstance(v, int) else int(v.data_ptr())
        rec.off[i] = int(kw.get(f'{t.name}_extraOffset', 0))
        keep.append(v)
      rec.num_elements = int(kw['numElements'])
      fl = kw.get('flags')
      rec.flags = None if fl is None else int(fl.data_ptr())
      if fl is not None:
        keep.append(fl)
      counts.append(int(kw['numElements']))
    raw = bytes(recs)
    dev_args = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to('cuda')
    items = self.work_items(counts)
    dev_items = torch.tensor(items if items else [(0, 0)], dtype=torch.int32, device='cuda').contiguous()
    counter = torch.zeros(1, dtype=torch.int32, device='cuda')
    return GroupedLaunch(self, dev_args, dev_items, len(items), counter, keep)

  def prepare_per_group(self, group_kwargs, streams=4):
    """The same argument sets as `prepare`, launched group by group through each
    generator's own launcher on `streams` side streams. Returns a `PerGroupLaunch`."""
    from .runtime import compile_generator
    if len(group_kwargs) != len(self.gens):
      raise ValueError('one argument set per group is required')
    return PerGroupLaunch([compile_generator(g) for g in self.gens], group_kwargs, streams)


class PerGroupLaunch:
  """The same mixed-shape batch with every group through its own launcher (the planner's
  own plan for its shape: prefetch stage, CTA width, constant or shared A), the groups spread
  over side streams (largest work first, onto the least-loaded stream) and joined back on the
  caller's stream; `capture()` records fork, launches and join in one CUDA graph.

  Against the persistent kernel it gives up the single launch and the shared work table (all
  groups there run one CTA shape, without the prefetch stage) for per-shape kernels.
  """

  def __init__(self, kernels, group_kwargs, streams):
    self.kernels = kernels
    self.kwargs = [dict(kw) for kw in group_kwargs]
    work = [int(kw['numElements']) * k.generator.get_chain().nz_flops_per_element()
            for k, kw in zip(kernels, group_kwargs)]
    load = [0] * max(1, streams)
    self.lanes = [[] for _ in load]
    for gid in sorted(range(len(kernels)), key=lambda i: -work[i]):
      lane = min(range(len(load)), key=lambda i: load[i])
      self.lanes[lane].append(gid)
      load[lane] += work[gid]
    self.streams = None
    self.graph = None

  def launch(self, stream=None):
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    if self.streams is None:
      self.streams = [torch.cuda.Stream() for _ in self.lanes]
    used = []
    for side, gids in zip(self.streams, self.lanes):
      gids = [g for g in gids if int(self.kwargs[g]['numElements']) > 0]
      if not gids:
        continue
      side.wait_stream(st)
      for gid in gids:
        self.kernels[gid](**dict(self.kwargs[gid], streamPtr=side.cuda_stream))
      used.append(side)
    for side in used:
      st.wait_stream(side)

  def capture(self):
    """Record the launch in a CUDA graph (after one eager launch for first-call setup)."""
    import torch
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
      self.launch(s)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
      self.launch(torch.cuda.current_stream())
    self.graph = g
    return g

  def replay(self):
    if self.graph is None:
      self.capture()
    self.graph.replay()


def host_records(kernel, group_kwargs):
  """tfb_group_args records in host memory (for the allocation-free entry point)."""
  recs = (_GroupArgs * len(group_kwargs))()
  for gid, (g, kw) in enumerate(zip(kernel.gens, group_kwargs)):
    rec = recs[gid]
    for i, (t, _) in enumerate(g.abi_symbols()):
      v = kw[t.name]
      rec.ptr[i] = v if isinstance(v, int) else int(v.data_ptr())
      rec.off[i] = int(kw.get(f'{t.name}_extraOffset', 0))
    rec.num_elements = int(kw['numElements'])
    fl = kw.get('flags')
    rec.flags = None if fl is None else int(fl.data_ptr())
  return recs


def launch_noalloc(kernel, group_kwargs, stream=None):
  """Call tfb_grouped_launch_noalloc_<set>: no device allocation by this call or the library."""
  import torch
  kernel._load()
  fn = getattr(kernel._lib, f'tfb_grouped_launch_noalloc_{kernel.name}')
  fn.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
  fn.restype = ctypes.c_int
  recs = host_records(kernel, group_kwargs)
  st = stream if stream is not None else torch.cuda.current_stream()
  rc = fn(ctypes.addressof(recs), len(group_kwargs), st.cuda_stream)
  if rc != 0:
    raise RuntimeError(f'allocation-free grouped launch failed with CUDA error {rc}')


class GroupedLaunch:
  """A prepared grouped launch; `launch()` runs it, `capture()` records it in a CUDA graph."""

  def __init__(self, kernel, dev_args, dev_items, num_items, counter, keep):
    self.kernel = kernel
    self.dev_args = dev_args
    self.dev_items = dev_items
    self.num_items = num_items
    self.counter = counter
    self._keep = keep
    self.graph = None

  def launch(self, stream=None):
    import torch
    fn = self.kernel._load()
    st = stream if stream is not None else torch.cuda.current_stream()
    rc = fn(self.dev_args.data_ptr(), self.dev_items.data_ptr(), self.num_items, self.counter.data_ptr(),
            st.cuda_stream)
    if rc != 0:
      raise RuntimeError(f'grouped launch failed with CUDA error {rc}')

  def capture(self):
    """Record launch (counter reset + persistent kernel) in a CUDA graph; returns the graph."""
    import torch
    self.kernel._load()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
      self.launch(s)            # warm-up outside capture (first-call attributes)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
      self.launch(torch.cuda.current_stream())
    self.graph = g
    return g

  def replay(self):
    if self.graph is None:
      self.capture()
    self.graph.replay()
