"""Benchmark: fused order-6 volume chain, elements/s on B200 (one JSON line on rank 0).

Workload: out_e(56x9) = sum_{t=0..2} K_t(56x56) * Q_e(56x9) * S_{e,t}(9x9),
K_t shared and sparse (seeded Bernoulli(0.45) pattern, ~1411 nonzeros), S_{e,t} per
element with 24 seeded nonzeros stored compactly at the start of a strided 81-value slot,
Q/out strided, uniform[-1,1] synthetic values, 500,000 elements per GPU (inputs of 2.2 GB,
larger than L2, so no flush is needed between steps). One step = one launch of the
generated kernel over all elements. The chain is generated through the public frontend
(`Generator`) and called through the emitted C-ABI launcher.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--variant auto|plain|tf32x3|bf16x3|tf32x3_form_b|...] [--elements E]
                  [--workload chain_o6|ew_update|mixed] [--basis B --quantities Q]

`--workload ew_update` measures the elementwise stage alone instead (its own JSON line);
`--workload mixed` one group of the mixed-shape workload (84 x 27 by default).

For N > 1 the driver launches one process per GPU (torchrun); elements are independent, so
each rank runs its own 500,000 elements (weak scaling) with no collective on the data
path; the time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'order-6 chain elements/s: split-TC vs plain FP32, same B200, rel err≤1e-6'
CASE = 'chain_o6'
WORKLOAD = 'order-6 volume chain: out(56x9) = sum_3 K(56x56, 45% sparse) Q(56x9) S(9x9, 24 nnz), FP32'
FALLBACK_HBM = 6650.0
# Elements per call of the reference's OpenMP kernel in both CPU legs (the `cpu_baseline`
# of the headline line and every step of `--impl reference`): a bounded sample of the
# 500,000-element workload, ~1.3 s per call on 16 host cores.
CPU_SAMPLE = 4096


def log(*a):
  print(*a, file=sys.stderr, flush=True)


def peaks():
  path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
  if os.path.exists(path):
    with open(path) as f:
      p = json.load(f)
    return p, 'measured'
  return {'hbm_gbs': FALLBACK_HBM, 'bf16_tflops': 1590.0}, 'fallback'


class Clocks:
  """nvidia-smi sampler over the timed region."""

  def __init__(self, index=0):
    self.index = index
    self.proc = None
    import tempfile
    self.path = os.path.join(tempfile.gettempdir(), f'tfb_clocks_{os.getpid()}_{index}.csv')

  def __enter__(self):
    os.makedirs(os.path.dirname(self.path), exist_ok=True)
    q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
    try:
      self.f = open(self.path, 'w')
      self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={q}',
                                    '--format=csv,noheader,nounits', '-lms', '100'],
                                   stdout=self.f, stderr=subprocess.DEVNULL)
      time.sleep(0.3)
    except (OSError, FileNotFoundError):
      self.proc = None
    return self

  def __exit__(self, *a):
    if self.proc is not None:
      time.sleep(0.2)
      self.proc.terminate()
      self.proc.wait()
      self.f.close()
      self._summary = self._read()
      try:
        os.remove(self.path)
      except OSError:
        pass

  def summary(self):
    return getattr(self, '_summary', None)

  def _read(self):
    if self.proc is None or not os.path.exists(self.path):
      return None
    mhz, mx, reasons = [], 0, set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
    for line in open(self.path):
      p = [x.strip() for x in line.split(',')]
      if len(p) < 9:
        continue
      try:
        mhz.append(float(p[1]))
        mx = max(mx, float(p[2]))
      except ValueError:
        continue
      for n, v in zip(names, p[5:9]):
        if v.lower() == 'active':
          reasons.add(n)
    if not mhz:
      return None
    return {'sm_mhz': statistics.median(mhz), 'sm_max_mhz': mx, 'reasons': sorted(reasons), 'samples': len(mhz)}


# ----------------------------------------------------------------------------- data

def make_inputs(gen, n, device, seed, dist='uniform', dtype=None):
  """Device buffers in the launcher's ABI layout for the order-6 chain.

  dist 'uniform': U(-1, 1); 'loguniform': random sign times 10^U(-3, 3) (magnitudes over
  six decades, the precision workload)."""
  import torch
  g = torch.Generator(device=device)
  g.manual_seed(seed)
  dtype = dtype or torch.float32

  def values(size):
    if dist == 'loguniform':
      mag = torch.pow(10.0, torch.rand(size, generator=g, device=device, dtype=torch.float64) * 6 - 3)
      sign = torch.where(torch.rand(size, generator=g, device=device) < 0.5, -1.0, 1.0).double()
      return (mag * sign).to(dtype)
    return (torch.rand(size, generator=g, device=device, dtype=dtype) * 2 - 1)
  bufs = {}
  for t, stype in gen.abi_symbols():
    if t.addressing.name == 'NONE':
      bufs[t.name] = values(t.spp.count_nz())
    else:
      bufs[t.name] = values(n * t.get_real_volume())
  return bufs


def kernel_error(k, gen):
  """Error word of a generated tensor-core kernel (a bounded wait that ran out), read and
  cleared; 0 for kernels without one."""
  import ctypes
  f = getattr(ctypes.CDLL(k.so_path), f'tfb_kernel_error_{gen.get_base_name()}', None)
  if f is None:
    return 0
  f.argtypes = [ctypes.c_void_p]
  f.restype = ctypes.c_int
  return int(f(None))


def check_accuracy(descrs, gen, bufs, n_check):
  """Relative-L2 and max-abs error of the first n_check elements vs the FP64 oracle."""
  import numpy as np
  from oracle.multilinear import Memory, evaluate
  mem = Memory()
  outname = None
  for t, _ in gen.abi_symbols():
    b = bufs[t.name]
    if t.addressing.name == 'NONE':
      mem.buffers[t.name] = b.double().cpu().numpy()
      continue
    vol = t.get_real_volume()
    mem.buffers[t.name] = b[:n_check * vol].double().cpu().numpy().copy()
    mem.starts[t.name] = np.arange(n_check, dtype=np.int64) * vol
    if t.direction.name != 'SOURCE':
      outname = t.name
  got = mem.buffers[outname].copy()
  evaluate(descrs, mem, n_check)
  ref = mem.buffers[outname]
  rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
  return {'rel_l2': rel, 'max_abs': float(np.abs(got - ref).max()), 'ref_max_abs': float(np.abs(ref).max()),
          'elements_checked': n_check}


def time_launches(fn, stream, steps, warmup, dist=None):
  """Run warmup untimed steps, then `steps` timed ones; per-launch and total times (ms)."""
  import torch
  for _ in range(warmup):
    fn()
  torch.cuda.synchronize()
  if dist is not None:
    dist.barrier()
  torch.cuda.synchronize()
  evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
  t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  t0.record(stream)
  for s, e in evs:
    s.record(stream)
    fn()
    e.record(stream)
  t1.record(stream)
  torch.cuda.synchronize()
  if dist is not None:
    dist.barrier()
  torch.cuda.synchronize()
  per = [s.elapsed_time(e) for s, e in evs]
  return t0.elapsed_time(t1), per


def link_bound(h2d_bytes, d2h_bytes, steps=3):
  """Host<->device link bound of one end-to-end step: `h2d_bytes` from pinned host memory
  and `d2h_bytes` back to pinned host memory, each as one contiguous copy, both directions
  at once on two streams and each direction alone (best of `steps`, ms)."""
  import torch
  hin = torch.empty(h2d_bytes, dtype=torch.uint8, pin_memory=True)
  din = torch.empty(h2d_bytes, dtype=torch.uint8, device='cuda')
  hout = torch.empty(d2h_bytes, dtype=torch.uint8, pin_memory=True)
  dout = torch.zeros(d2h_bytes, dtype=torch.uint8, device='cuda')
  s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
  cur = torch.cuda.current_stream()

  def run(do_in, do_out):
    best = None
    for _ in range(steps + 1):
      torch.cuda.synchronize()
      t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      t0.record(cur)
      for on, st, dst, src in ((do_in, s_in, din, hin), (do_out, s_out, hout, dout)):
        if on:
          st.wait_event(t0)
          with torch.cuda.stream(st):
            dst.copy_(src, non_blocking=True)
          cur.wait_stream(st)
      t1.record(cur)
      torch.cuda.synchronize()
      ms = t0.elapsed_time(t1)
      best = ms if best is None else min(best, ms)
    return best

  run(True, True)
  duplex, h2d_ms, d2h_ms = run(True, True), run(True, False), run(False, True)
  return {'duplex_ms': duplex, 'h2d_alone_gbs': h2d_bytes / h2d_ms / 1e6, 'd2h_alone_gbs': d2h_bytes / d2h_ms / 1e6,
          'duplex_h2d_gbs': h2d_bytes / duplex / 1e6, 'duplex_d2h_gbs': d2h_bytes / duplex / 1e6}


# ----------------------------------------------------------------------------- CPU baseline

def _cpu_bench(args_list):
  """Run oracle/cpu_bench.py in a fresh interpreter (system OpenMP runtime) and parse its JSON."""
  cmd = [sys.executable, '-m', 'oracle.cpu_bench'] + args_list
  env = dict(os.environ)
  env['OMP_TARGET_OFFLOAD'] = 'DISABLED'  # the CPU baseline never runs on an offload device
  proc = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, env=env, timeout=900)
  if proc.returncode != 0:
    log(proc.stderr[-2000:])
    return None
  return json.loads(proc.stdout.strip().splitlines()[-1])


def reference_cpu(steps=3):
  """The reference's OpenMP-backend chain kernel on all host cores: `steps` calls of
  CPU_SAMPLE elements after one warm-up call (mean rate)."""
  from oracle import baseline
  tag = 'bench_chain_o6_float'
  if not baseline.available(tag):
    return None
  r = _cpu_bench(['--tag', tag, '--case', CASE, '--fixed', str(CPU_SAMPLE), '--steps', str(steps), '--warmup', '1'])
  if r is None:
    return None
  return {'value': r['elements_per_s'], 'unit': 'elements/s', 'cores': r['cores'], 'kind': 'reference',
          'sample': f'{CPU_SAMPLE} elements of the 500,000-element workload per call, mean of {steps} calls '
                    f'after one warm-up, reference OpenMP-backend kernel (g++ -O3 -march=native -fopenmp, '
                    f'host fallback) on all host threads'}


def reference_cpu_c0(n=10000, steps=5):
  """Config 0 as the reference runs it: its OpenMP-backend GEMM kernel (56x56 * 56x9,
  pointer arrays, 10,000 elements: the full workload), median of `steps` calls after one
  warm-up, all host cores."""
  from oracle import baseline
  tag = 'bench_c0_gemm_ptr_float'
  if not baseline.available(tag):
    return None
  r = _cpu_bench(['--tag', tag, '--case', 'c0_gemm_ptr', '--fixed', str(n), '--steps', str(steps), '--warmup', '1'])
  if r is None:
    return None
  return {'value': r['elements_per_s_median'], 'unit': 'elements/s', 'cores': r['cores'], 'kind': 'reference',
          'median_s': r['median_s'],
          'sample': f'the full {n}-element workload per call, median of {steps} calls after one warm-up, '
                    'reference OpenMP-backend kernel on all host threads'}


def reference_cpu_mixed(groups, sample=512, steps=3):
  """Config 3 on the host: the reference's OpenMP-backend kernel of every group (one
  launcher per shape, as the reference runs mixed shapes), each timed on `sample`
  elements (mean of `steps` calls after one warm-up); the workload's time is the sum over
  groups of elements / rate."""
  from oracle import baseline
  per, total_s, total_el, cores = [], 0.0, 0, None
  for b, q, n in groups:
    tag = baseline.mixed_tag(b, q)
    if not baseline.available(tag):
      return None
    r = _cpu_bench(['--tag', tag, '--case', f'mixed_{b}_{q}', '--fixed', str(sample), '--steps', str(steps),
                    '--warmup', '1'])
    if r is None:
      return None
    cores = r['cores']
    per.append({'basis': b, 'quantities': q, 'elements_per_s': r['elements_per_s'], 'elements': n,
                'workload_s': n / r['elements_per_s']})
    total_s += n / r['elements_per_s']
    total_el += n
  return {'value': total_el / total_s, 'unit': 'elements/s', 'cores': cores, 'kind': 'reference',
          'workload_s': total_s, 'per_group': per,
          'sample': f'{sample} elements per group and call, mean of {steps} calls after one warm-up, '
                    'reference OpenMP-backend kernel of each group on all host threads; workload time = '
                    'sum over groups of elements / rate'}


def impl_reference(args, rank, world):
  if rank != 0:
    return
  from oracle import baseline
  tag = 'bench_chain_o6_float'
  if not baseline.available(tag):
    print(json.dumps({'impl': 'reference', 'unavailable': 'reference OpenMP build missing (oracle/_ref)'}))
    return
  n = CPU_SAMPLE
  r = _cpu_bench(['--tag', tag, '--case', CASE, '--fixed', str(n), '--steps', str(args.steps),
                  '--warmup', str(args.warmup)])
  if r is None:
    print(json.dumps({'impl': 'reference', 'unavailable': 'reference OpenMP kernel failed to run'}))
    return
  ms = 1e3 * sum(r['times']) / len(r['times'])
  value = r['elements_per_s']
  line = {
    'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'elements/s', 'n_gpus': world,
    'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
    'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
    'config': {'workload': WORKLOAD,
               'elements_per_step': n, 'full_workload_elements': args.elements},
    'cpu_baseline': {'value': value, 'unit': 'elements/s', 'cores': r['cores'], 'kind': 'reference',
                     'sample': f'{n} elements per step (bounded sample of the {args.elements}-element workload), '
                               'reference OpenMP-backend kernel on all host threads'},
    'e2e': {'value': value, 'unit': 'elements/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
  }
  print(json.dumps(line))


# ----------------------------------------------------------------------------- ours

_FP32_PEAK = []


def fp32_peak_cached():
  """FP32 FFMA peak measured once per run (the probe of the native runtime library)."""
  if not _FP32_PEAK:
    from tensorforge_b200.runtime.peaks import fma_peak
    _FP32_PEAK.append(fma_peak('float'))
  return _FP32_PEAK[0]


def extra_workloads(stream, short=False, cpu=True):
  """Secondary BASELINE configs measured next to the headline (device-resident inputs);
  with `cpu`, the reference's OpenMP-backend kernels for configs 0 and 3 on the host."""
  import torch
  from tensorforge_b200 import workloads as cases
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  out = {}
  dev = torch.device('cuda')
  # config 0: C_e = A * B_e, 56x56 * 56x9, pointer arrays
  for n in ((10000,) if short else (10000, 1000000)):
    g = make('c0_gemm_ptr', 'float')
    k = compile_generator(g)
    sym = {t.name: t for t, _ in g.abi_symbols()}
    kw = {'numElements': n}
    keep = []
    for name, t in sym.items():
      if t.addressing.name == 'NONE':
        kw[name] = torch.rand(t.get_real_volume(), device=dev)
      else:
        buf = torch.rand(n * 504, device=dev)
        ptrs = buf.data_ptr() + torch.arange(n, device=dev, dtype=torch.int64) * 504 * 4
        keep.append(buf)
        kw[name] = ptrs
    total, per = time_launches(lambda: k(**kw), stream, 10, 3)
    ms = sum(per) / len(per)
    flops = n * g.get_chain().nz_flops_per_element()
    # both bounds: FP32 pipe (56,448 flops per element) and HBM (4,048 bytes: B, C, 2 pointers)
    bytes_el = g.get_chain().bytes_per_element()
    fp32 = fp32_peak_cached()
    hbm = peaks()[0]['hbm_gbs'] * 1e9
    out[f'c0_gemm_{n}'] = {'elements_per_s': n / (ms / 1e3), 'gflops': flops / (ms / 1e3) / 1e9, 'ms': ms,
                           'plan': g.get_plan().key(),
                           'roofline': {'fp32_bound_el_s': fp32 / (flops / n), 'hbm_bound_el_s': hbm / bytes_el,
                                        'frac_of_tighter': (n / (ms / 1e3)) / min(fp32 / (flops / n), hbm / bytes_el),
                                        'bytes_per_element': bytes_el, 'flops_per_element': flops / n}}
    if n == 10000 and cpu:
      out[f'c0_gemm_{n}']['cpu_baseline'] = reference_cpu_c0(n)
    if n >= 1000000:
      # the same GEMM on the tensor cores (TF32x3: operand form B, the default for one term,
      # and form U; parity in the GPU tests)
      tc = {}
      for label, variant in (('tf32x3', None), ('tf32x3_form_u', {'form': 'u'})):
        gt = make('c0_gemm_ptr', 'float', precision='tf32x3', **({'variant': variant} if variant else {}))
        kt = compile_generator(gt)
        total, per = time_launches(lambda: kt(**kw), stream, 10, 3)
        mt = sum(per) / len(per)
        tc[label] = {'elements_per_s': n / (mt / 1e3), 'plan': gt.get_plan().key(),
                     'frac_hbm': (n / (mt / 1e3)) / (hbm / bytes_el)}
      out[f'c0_gemm_{n}']['tensor_cores'] = tc
  # config 3: mixed shapes, one persistent launch over a work table, replayed from a CUDA graph
  from tensorforge_b200.kernels import grouped_catalogue
  gk = dict(grouped_catalogue())['bench_c3']
  groups = cases.mixed_shape_groups()
  kws, total_el, nz = [], 0, 0.0
  for g, (b, q, n) in zip(gk.gens, groups):
    kw = {'numElements': n}
    for t, _ in g.abi_symbols():
      size = t.spp.count_nz() if t.addressing.name == 'NONE' else n * t.get_real_volume()
      kw[t.name] = torch.rand(size, device=dev) * 2 - 1
    kws.append(kw)
    total_el += n
    nz += n * g.get_chain().nz_flops_per_element()
  launch = gk.prepare(kws)
  launch.capture()
  total, per = time_launches(launch.replay, stream, 10, 3)
  ms = sum(per) / len(per)
  sep = [compile_generator(g) for g in gk.gens]

  def separate():
    for k, kw in zip(sep, kws):
      k(**kw)
  total2, per2 = time_launches(separate, stream, 5, 2)
  ms2 = sum(per2) / len(per2)
  # the same batch as one CUDA graph of per-group kernels on 4 side streams
  pg = gk.prepare_per_group(kws, streams=4)
  pg.capture()
  _, per3 = time_launches(pg.replay, stream, 10, 3)
  ms3 = sum(per3) / len(per3)
  per_group = []
  fp32 = fp32_peak_cached()
  hbm = peaks()[0]['hbm_gbs'] * 1e9
  bound_s = 0.0
  for i, (b, q, n) in enumerate(groups):  # the same launch with every other group emptied
    one = gk.prepare([dict(kw, numElements=(kw['numElements'] if j == i else 0)) for j, kw in enumerate(kws)])
    _, pg = time_launches(one.launch, stream, 3, 1)
    g_ms = sum(pg) / len(pg)
    ch = gk.gens[i].get_chain()
    g_nz = n * ch.nz_flops_per_element()
    g_bytes = n * ch.bytes_per_element() + sum(o.storage_size() * 4 for o in ch.shared())
    # roofline time of the group: the slower of its FP32-pipe time (nz flops) and HBM time
    g_bound = max(g_nz / fp32, g_bytes / hbm)
    bound_s += g_bound
    # the same group through its own launcher (the planner's plan for its shape)
    _, ps = time_launches(lambda i=i: sep[i](**kws[i]), stream, 3, 1)
    s_ms = sum(ps) / len(ps)
    per_group.append({'basis': b, 'quantities': q, 'elements': n, 'ms': g_ms, 'elements_per_s': n / (g_ms / 1e3),
                      'nz_gflops': g_nz / (g_ms / 1e3) / 1e9,
                      'standalone_ms': s_ms, 'standalone_plan': gk.gens[i].get_plan().key(),
                      'roofline': {'bound': 'fp32' if g_nz / fp32 >= g_bytes / hbm else 'hbm',
                                   'frac': g_bound / (g_ms / 1e3), 'fp32_frac': g_nz / fp32 / (g_ms / 1e3),
                                   'hbm_frac': g_bytes / hbm / (g_ms / 1e3)}})
  out['c3_mixed_shapes'] = {'elements': total_el, 'groups': len(groups), 'elements_per_s': total_el / (ms / 1e3),
                            'nz_gflops': nz / (ms / 1e3) / 1e9, 'ms': ms, 'launch': 'one persistent kernel, CUDA graph replay',
                            'separate_launches_ms': ms2, 'separate_elements_per_s': total_el / (ms2 / 1e3),
                            'graph_per_group_ms': ms3, 'graph_per_group_elements_per_s': total_el / (ms3 / 1e3),
                            'graph_per_group': 'one CUDA graph: each group through its own launcher, 4 side streams',
                            'per_group': per_group,
                            'roofline': {'bound': 'sum over groups of max(nz flops / FP32 peak, bytes / HBM)',
                                         'bound_ms': bound_s * 1e3, 'frac_persistent': bound_s / (ms / 1e3),
                                         'frac_graph_per_group': bound_s / (ms3 / 1e3),
                                         'fp32_peak_tflops': fp32 / 1e12, 'hbm_gbs': hbm / 1e9,
                                         'peak_source': 'FP32: FFMA probe of this run; HBM: measured copy bandwidth'}}
  if cpu:
    out['c3_mixed_shapes']['cpu_baseline'] = reference_cpu_mixed(groups)
  # config 4: the shipped cost model on held-out chains of the seeded tuning set, every
  # variant re-measured here (the exhaustive tuner's timings), bounded in time
  from tensorforge_b200.tune import heldout, select
  t4 = time.time()
  recs = heldout.measure_all(heldout.build_all(heldout.heldout_specs(40)), time_limit=20 if short else 60)
  c4 = heldout.summary(heldout.score(recs, select.predict))
  c4.update({'chains_requested': 40, 'seconds': time.time() - t4, 'inference': select.last_inference,
             'regret': '(measured time of pick - measured best) / measured best; default = the planner '
                       'without the cost model; chains from the 20 % test split of the 2,000-chain set'})
  out['c4_cost_model'] = c4
  # config 2: log-uniform magnitudes through every precision variant, error vs the FP64 oracle
  descrs = cases.build(CASE, cases.ns_from_module('tensorforge_b200'))
  n2 = 100000 if short else 500000
  c2 = {}
  for label, fp, opts in (('fp32_plain', 'float', {}), ('tf32x3', 'float', {'precision': 'tf32x3'}),
                          ('bf16x3', 'float', {'precision': 'bf16x3'}),
                          ('fp64_colprog', 'double', {'variant': {'strategy': 'colprog'}}),
                          ('fp64_dmma', 'double', {})):
    g = make(CASE, fp, **opts)
    k = compile_generator(g)
    kw = make_inputs(g, n2, dev, 7, 'loguniform', torch.float64 if fp == 'double' else torch.float32)
    kw['numElements'] = n2
    k(**kw)
    torch.cuda.synchronize()
    acc = check_accuracy(descrs, g, kw, 2048)
    total, per = time_launches(lambda: k(**kw), stream, 5, 2)
    ms = sum(per) / len(per)
    c2[label] = {'elements_per_s': n2 / (ms / 1e3), 'plan': g.get_plan().key(), 'rel_l2': acc['rel_l2'],
                 'max_abs': acc['max_abs'], 'ref_max_abs': acc['ref_max_abs']}
    del kw
  out['c2_precision_loguniform'] = {'elements': n2, 'values': 'sign * 10^U(-3,3), seed 7', 'variants': c2}
  torch.cuda.empty_cache()
  # elementwise stage: pointwise nonlinear update of a 56x9 block per element (HBM bound)
  from tensorforge_b200.kernels import EW_BENCH_VARIANTS
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  ns = cases.ns_from_module('tensorforge_b200')
  n = 200000 if short else 1000000
  hbm = peaks()[0]['hbm_gbs']
  ew = {}
  bufs = {}
  for v in [None] + EW_BENCH_VARIANTS:
    g = Generator(cases.build_elementwise('ew_update', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT,
                                                                    Options(variant=v)))
    g.generate()
    k = compile_generator(g)
    if not bufs:
      for t, _ in g.abi_symbols():
        bufs[t.name] = 0.5 if t.addressing.name == 'SCALAR' else torch.rand(n * t.get_real_volume(), device=dev) * 2 - 1
    kw = dict(bufs, numElements=n)
    total, per = time_launches(lambda: k(**kw), stream, 5, 2)
    ms = sum(per) / len(per)
    gbs = n * g.get_chain().bytes_per_element() / (ms / 1e3) / 1e9
    ew['default' if v is None else g.get_plan().key()] = {
      'elements_per_s': n / (ms / 1e3), 'ms': ms, 'hbm_gbs': gbs, 'frac_hbm': gbs / hbm, 'plan': g.get_plan().key()}
  out['elementwise_update'] = {'elements': n, 'bytes_per_element': 2 * 504 * 4, 'peak_hbm_gbs': hbm,
                               'statements': 't = Q*s; O = t > 0 ? t*exp(-t*t) : 0.5*t (56x9, FP32)',
                               'variants': ew}
  bufs.clear()
  # the order-6 chain with a pointwise update fused as a column-program epilogue, next to
  # the same chain without it (both plain FP32 column programs)
  n = 100000 if short else 500000
  epi = {}
  for label, descrs in (('chain_only', cases.build(CASE, ns)), ('chain_with_epilogue',
                                                                cases.build_elementwise('ew_chain_epilogue', ns))):
    g = Generator(descrs, Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
    g.generate()
    k = compile_generator(g)
    kw = {'numElements': n}
    for t, _ in g.abi_symbols():
      if t.addressing.name == 'SCALAR':
        kw[t.name] = 0.5
      else:
        size = t.spp.count_nz() if t.addressing.name == 'NONE' else n * t.get_real_volume()
        kw[t.name] = torch.rand(size, device=dev) * 2 - 1
    total, per = time_launches(lambda: k(**kw), stream, 5, 2)
    ms = sum(per) / len(per)
    epi[label] = {'elements_per_s': n / (ms / 1e3), 'ms': ms, 'plan': g.get_plan().key(),
                  'bytes_per_element': g.get_chain().bytes_per_element()}
    del kw
  out['elementwise_epilogue'] = {'elements': n, 'statements': 'out = out > 0 ? out : 0.1*out; out = out + P*s',
                                 'variants': epi}
  torch.cuda.empty_cache()
  # FP64 order-6 chain
  n = 100000 if short else 500000
  for label, opts in (('fp64_colprog', {'variant': {'strategy': 'colprog'}}), ('fp64_dmma', {})):
    g = make(CASE, 'double', **opts)
    k = compile_generator(g)
    kw = {'numElements': n}
    for t, _ in g.abi_symbols():
      size = t.spp.count_nz() if t.addressing.name == 'NONE' else n * t.get_real_volume()
      kw[t.name] = torch.rand(size, device=dev, dtype=torch.float64) * 2 - 1
    total, per = time_launches(lambda: k(**kw), stream, 5, 2)
    ms = sum(per) / len(per)
    out[f'chain_o6_{label}'] = {'elements_per_s': n / (ms / 1e3), 'plan': g.get_plan().key(), 'elements': n,
                                'nz_gflops': n * g.get_chain().nz_flops_per_element() / (ms / 1e3) / 1e9,
                                'hbm_gbs': n * g.get_chain().bytes_per_element() / (ms / 1e3) / 1e9}
  return out


def impl_ours(args, rank, world, dist):
  import torch
  from tensorforge_b200.runtime import ranks
  from tensorforge_b200 import workloads as cases
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  from tensorforge_b200.common.basic_types import DataFlowDirection
  device = torch.device('cuda', torch.cuda.current_device())
  n = args.elements
  variants = ['plain'] if args.variant == 'plain' else (
    [args.variant] if args.variant != 'auto' else ['tf32x3', 'plain', 'tf32x3_pipe2'])
  opts_of = {'plain': {}, 'tf32x3': {'precision': 'tf32x3'},
             'tf32x3_ahead': {'precision': 'tf32x3', 'variant': {'form': 'u', 'ahead': 1}},
             'tf32x3_pipe2': {'precision': 'tf32x3', 'variant': {'form': 'u', 'pipe': 2}},
             'tf32x3_s2': {'precision': 'tf32x3', 'variant': {'form': 'u', 'slots': 2}},
             'tf32x3_nl': {'precision': 'tf32x3', 'variant': {'form': 'u', 'loader': 0}},
             'tf32x3_u2': {'precision': 'tf32x3', 'variant': {'form': 'u', 'urows': 2}},
             'tf32x3_q': {'precision': 'tf32x3', 'variant': {'form': 'u', 'qreg': 1}},
             'tf32x3_q_s2': {'precision': 'tf32x3', 'variant': {'form': 'u', 'qreg': 1, 'slots': 2}},
             'tf32x3_loader': {'precision': 'tf32x3', 'variant': {'form': 'u', 'loader': 1}},
             'tf32x3_u2f': {'precision': 'tf32x3', 'variant': {'form': 'u', 'urows': 2, 'fuse': 1}},
             'tf32x3_qf': {'precision': 'tf32x3', 'variant': {'form': 'u', 'qreg': 1, 'fuse': 1}},
             'tf32x3_u2l': {'precision': 'tf32x3', 'variant': {'form': 'u', 'urows': 2, 'loader': 2}},
             'tf32x3_u2fl': {'precision': 'tf32x3', 'variant': {'form': 'u', 'urows': 2, 'fuse': 1, 'loader': 2}},
             'tf32x3_nf': {'precision': 'tf32x3', 'variant': {'form': 'u', 'fuse': 0}},
             'tf32x3_l3': {'precision': 'tf32x3', 'variant': {'form': 'u', 'loader': 3}},
             'tf32x3_spin': {'precision': 'tf32x3', 'variant': {'form': 'u', 'sleep': 0}},
             'tf32x3_sl1': {'precision': 'tf32x3', 'variant': {'form': 'u', 'sleep': 1}},
             'tf32x3_sl2': {'precision': 'tf32x3', 'variant': {'form': 'u', 'sleep': 2}},
             'tf32x3_ds': {'precision': 'tf32x3', 'variant': {'form': 'u', 'ostage': 0}},
             'tf32x3_op': {'precision': 'tf32x3', 'variant': {'form': 'u', 'opad': 1}},
             'tf32x3_nuw': {'precision': 'tf32x3', 'variant': {'form': 'u', 'uwarp': 0}},
             'tf32x3_dl': {'precision': 'tf32x3', 'variant': {'form': 'u', 'direct': 1}},
             'tf32x3_l64': {'precision': 'tf32x3', 'variant': {'form': 'u', 'l64': 1}},
             'tf32x3_oswz': {'precision': 'tf32x3', 'variant': {'form': 'u', 'oswz': 1}},
             'tf32x3_estg': {'precision': 'tf32x3', 'variant': {'form': 'u', 'estg': 1}},
             'tf32x3_nlpk': {'precision': 'tf32x3', 'variant': {'form': 'u', 'lpk': 0}},
             'tf32x3_nepk': {'precision': 'tf32x3', 'variant': {'form': 'u', 'epk': 0}},
             'tf32x3_sl3': {'precision': 'tf32x3', 'variant': {'form': 'u', 'sleep': 3}},

             'plain_rs2': {'variant': {'strategy': 'colprog', 'threads': 256, 'rsplit': 2, 'min_blocks': 2}},
             'tf32x3_form_b': {'precision': 'tf32x3', 'variant': {'form': 'b'}},
             'tf32x3_form_b2': {'precision': 'tf32x3', 'variant': {'form': 'b', 'bbuf': 2}},
             'tf32x3_form_b_ws': {'precision': 'tf32x3', 'variant': {'form': 'b', 'ws': 1}},
             'bf16x3': {'precision': 'bf16x3'}, 'generic': {'variant': {'strategy': 'generic'}}}
  results = {}
  stream = torch.cuda.current_stream()
  primary = None
  ref_gen = make(CASE, 'float')
  bufs = make_inputs(ref_gen, n, device, seed=ranks.rank_seed(1234, rank))
  outname = [t.name for t, _ in ref_gen.abi_symbols() if t.direction != DataFlowDirection.SOURCE][0]
  descrs = cases.build(CASE, cases.ns_from_module('tensorforge_b200'))
  extra = ['plain'] if 'plain' not in variants else []
  for name in variants + extra:
    try:
      gen = make(CASE, 'float', **opts_of[name])
    except Exception as e:  # variant not available for this chain
      log(f'variant {name} unavailable: {e}')
      continue
    if name.startswith(('tf32x3', 'bf16x3')) and gen.get_plan().strategy != 'tcsplit':
      log(f'variant {name} fell back to {gen.get_plan().strategy}; skipped')
      continue
    k = compile_generator(gen)
    kw = {t.name: bufs[t.name] for t, _ in gen.abi_symbols()}
    kw['numElements'] = n
    kw['streamPtr'] = stream.cuda_stream
    fn = lambda k=k, kw=kw: k(**kw)  # noqa: E731
    fn()
    torch.cuda.synchronize()
    acc = check_accuracy(descrs, gen, bufs, min(n, 2048))
    steps = args.steps if primary is None else max(3, args.steps // 2)
    total, per = time_launches(fn, stream, steps, max(3, args.warmup), dist if primary is None else None)
    err = kernel_error(k, gen)
    results[name] = {'kernel': gen.get_base_name(), 'plan': gen.get_plan().key(), 'ms_total': total,
                     'launch_ms': per, 'accuracy': acc, 'gen': gen, 'k': k, 'kw': kw}
    if err:
      # a bounded wait ran out: the timing is not the kernel's, the variant is not reported
      log(f'variant {name}: kernel error word {err} (a bounded wait ran out); not used')
      results[name]['kernel_error'] = err
    ok = (name == 'plain' or acc['rel_l2'] <= 1e-6) and not err
    if primary is None:
      # the choice changes the collective sequence (timed barriers): every rank must agree
      ok = ranks.all_ranks(ok, dist)
    if primary is None and ok:
      primary = name
    log(f'{name}: {n / (total / steps / 1e3):.3e} el/s, rel_l2 {acc["rel_l2"]:.2e}, plan {gen.get_plan().key()}')
  if primary is None:
    raise RuntimeError('no benchmark variant ran')
  pr = results[primary]
  k, kw, gen = pr['k'], pr['kw'], pr['gen']

  # the timed region of record: K steps of the primary variant, clocks sampled meanwhile
  with Clocks(index=torch.cuda.current_device()) as clocks:
    total, per = time_launches(lambda: k(**kw), stream, args.steps, args.warmup, dist)
  if kernel_error(k, gen):
    raise RuntimeError(f'{primary}: a bounded wait ran out during the timed region')
  ms = ranks.max_over_ranks(total / args.steps, dist)
  value = ranks.aggregate_rate(world, n, ms)

  # end to end through the C-ABI launcher with host buffers (pinned), copies inside the timed region
  host = {name: b.cpu().pin_memory() for name, b in bufs.items()}

  # slices of the batch flow through three streams: copy-in, kernel and copy-out overlap
  # (16 slices measured best of 8-64; compactly stored S operands are copied without the
  # unused tail of their slots)
  from tensorforge_b200.runtime.pipeline import HostPipeline
  pipe = HostPipeline(k, gen, slices=16, streams=3)
  inputs = [t.name for t, _ in gen.abi_symbols() if t.direction == DataFlowDirection.SOURCE]
  h2d = 0
  for t, _ in gen.abi_symbols():
    if t.name not in inputs:
      continue
    if t.name in pipe.used:
      h2d += n * pipe.used[t.name] * host[t.name].element_size()
    else:
      h2d += host[t.name].numel() * host[t.name].element_size()
  d2h = host[outname].numel() * host[outname].element_size()
  dev_bufs = {t.name: kw[t.name] for t, _ in gen.abi_symbols()}

  def e2e_step():
    pipe(host, dev_bufs, n)

  e_steps = max(2, min(args.steps, 5))
  e_total, _ = time_launches(e2e_step, stream, e_steps, 1, dist)
  e_ms = ranks.max_over_ranks(e_total / e_steps, dist)

  if rank != 0:
    return
  chain = gen.get_chain()
  bytes_el = chain.bytes_per_element()
  shared_bytes = sum(o.storage_size() * 4 for o in chain.shared())
  alg_bytes = n * bytes_el + shared_bytes
  mean_launch = sum(per) / len(per)
  pk, pk_src = peaks()
  achieved = alg_bytes / (mean_launch / 1e3) / 1e9
  traffic = None
  prof = os.path.join(ROOT, 'profiles', 'traffic.json')
  if os.path.exists(prof):
    with open(prof) as f:
      tr = json.load(f).get(pr['plan'])
    if tr is not None:
      traffic = tr['bytes_per_element'] * n
  roofline = {'bound': 'hbm', 'achieved': achieved, 'peak': pk['hbm_gbs'], 'unit': 'GB/s',
              'frac': achieved / pk['hbm_gbs'], 'traffic': traffic,
              'peak_source': f'{pk_src} HBM copy bandwidth', 'kernel': pr['kernel'],
              'algorithmic_bytes_per_launch': alg_bytes}
  nz = chain.nz_flops_per_element()
  plain = results.get('plain')
  extra_out = {}
  if plain is not None:
    p_launch = sum(plain['launch_ms']) / len(plain['launch_ms'])
    fp32_peak = fp32_peak_cached()
    p_flops = n * nz / (p_launch / 1e3)
    extra_out['plain_fp32'] = {
      'elements_per_s': n / (p_launch / 1e3), 'kernel': plain['kernel'], 'plan': plain['plan'],
      'accuracy': plain['accuracy'],
      'roofline': {'bound': 'fp32', 'achieved': p_flops / 1e12, 'peak': fp32_peak / 1e12, 'unit': 'TFLOP/s',
                   'frac': p_flops / fp32_peak, 'flops_per_element': nz,
                   'dense_equivalent_flops_per_element': chain.dense_flops_per_element(),
                   'peak_source': 'measured FP32 FFMA probe (libtfb200_runtime tfb_fma_peak_launch), same run'}}
  for name, r in results.items():
    extra_out.setdefault('variants', {})[name] = {
      'elements_per_s': n / (sum(r['launch_ms']) / len(r['launch_ms']) / 1e3), 'plan': r['plan'],
      'rel_l2': r['accuracy']['rel_l2'], 'max_abs': r['accuracy']['max_abs'],
      **({'kernel_error': r['kernel_error']} if 'kernel_error' in r else {})}
  # the link bound of the end-to-end step (contiguous copies of the same byte counts)
  link = link_bound(h2d, d2h)
  link['frac'] = link['duplex_ms'] / e_ms
  cpu = reference_cpu() if (world == 1 and not args.no_cpu) else None
  extras = (extra_workloads(stream, short=args.no_cpu, cpu=not args.no_cpu)
            if (world == 1 and not args.no_extras) else None)
  line = {
    'metric': METRIC, 'value': value, 'unit': 'elements/s', 'n_gpus': world, 'steps': args.steps,
    'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
    'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
    'config': {'workload': WORKLOAD,
               'elements_per_gpu': n, 'variant': primary, 'plan': pr['plan'],
               'l2': 'inputs larger than L2 (no flush)'},
    'accuracy': pr['accuracy'],
    'roofline': roofline,
    'cpu_baseline': cpu,
    'e2e': {'value': world * n / (e_ms / 1e3), 'unit': 'elements/s', 'h2d_bytes_per_step': h2d,
            'd2h_bytes_per_step': d2h, 'api': 'runtime.pipeline.HostPipeline (16 slices, 3 streams)',
            'link_bound': link},
    'gpu_launches': args.steps,
    'clocks': clocks.summary(),
  }
  line.update(extra_out)
  if extras is not None:
    line['other_configs'] = extras
  print(json.dumps(line))


def impl_elementwise(args):
  """`--workload ew_update`: the elementwise stage alone (t = Q*s; O = t > 0 ? t*exp(-t*t) :
  0.5*t over a 56x9 block per element), default plan, device-resident inputs larger than L2;
  the oracle timed on a bounded host sample as the CPU figure (the reference cannot emit
  this path)."""
  import numpy as np
  import torch
  from tensorforge_b200 import workloads as cases
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  torch.cuda.set_device(0)
  ns = cases.ns_from_module('tensorforge_b200')
  n = args.elements
  g = Generator(cases.build_elementwise('ew_update', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
  g.generate()
  k = compile_generator(g)
  dev = torch.device('cuda')
  kw = {'numElements': n}
  for t, _ in g.abi_symbols():
    kw[t.name] = 0.5 if t.addressing.name == 'SCALAR' else torch.rand(n * t.get_real_volume(), device=dev) * 2 - 1
  stream = torch.cuda.current_stream()
  with Clocks(index=torch.cuda.current_device()) as clocks:
    total, per = time_launches(lambda: k(**kw), stream, args.steps, max(3, args.warmup))
  ms = total / args.steps
  launch = sum(per) / len(per)
  bytes_el = g.get_chain().bytes_per_element()
  pk, pk_src = peaks()
  achieved = n * bytes_el / (launch / 1e3) / 1e9
  # CPU: the oracle (numpy, FP64) on a bounded sample
  from oracle import harness, multilinear
  sample = 2000
  descrs = cases.build_elementwise('ew_update', ns)
  lay, mem = harness.make_memory(descrs, sample, seed=1)
  t0 = time.perf_counter()
  reps = 0
  while time.perf_counter() - t0 < 3.0:
    multilinear.evaluate(descrs, mem, sample)
    reps += 1
  cpu_rate = reps * sample / (time.perf_counter() - t0)
  print(json.dumps({
    'metric': 'elementwise update throughput', 'value': n / (ms / 1e3), 'unit': 'elements/s', 'n_gpus': 1,
    'steps': args.steps, 'warmup': max(3, args.warmup), 'ms_per_step': ms, 'higher_is_better': True,
    'dtype': 'f32', 'data': 'synthetic',
    'config': {'workload': 'elementwise update, 56x9 block per element, FP32', 'elements': n,
               'plan': g.get_plan().key(), 'l2': 'inputs larger than L2 (no flush)'},
    'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': pk['hbm_gbs'], 'unit': 'GB/s',
                 'frac': achieved / pk['hbm_gbs'], 'traffic': None, 'bytes_per_element': bytes_el,
                 'peak_source': f'{pk_src} HBM copy bandwidth', 'kernel': g.get_base_name()},
    'cpu_baseline': {'value': cpu_rate, 'unit': 'elements/s', 'cores': 1, 'kind': 'port',
                     'sample': f'{sample} elements through the numpy FP64 oracle, repeated for 3 s'},
    'gpu_launches': args.steps, 'clocks': clocks.summary()}))


def impl_mixed_group(args):
  """`--workload mixed`: one group of the mixed-shape workload alone (basis x quantities,
  three sparse basis x basis K terms at 45 %, a sparse quantity x quantity S per element and
  term) under its default plan, device-resident inputs; FP32 roofline on the nz flops with
  the FMA probe of the same run; error of the first 256 elements against the FP64 oracle."""
  import torch
  from tensorforge_b200 import workloads as cases
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  torch.cuda.set_device(0)
  ns = cases.ns_from_module('tensorforge_b200')
  n, b, q = args.elements, args.basis, args.quantities
  g = Generator(cases.mixed_chain(ns, b, q), Context('sm_100a', 'cuda', FloatingPointType.FLOAT))
  g.generate()
  k = compile_generator(g)
  bufs = make_inputs(g, n, torch.device('cuda'), seed=1)
  kw = {t.name: bufs[t.name] for t, _ in g.abi_symbols()}
  kw['numElements'] = n
  k(**kw)
  torch.cuda.synchronize()
  acc = check_accuracy(cases.mixed_chain(ns, b, q), g, bufs, min(n, 256))
  stream = torch.cuda.current_stream()
  with Clocks(index=torch.cuda.current_device()) as clocks:
    total, per = time_launches(lambda: k(**kw), stream, args.steps, max(3, args.warmup))
  launch = sum(per) / len(per)
  nz = g.get_chain().nz_flops_per_element()
  peak = fp32_peak_cached()
  flops = n * nz / (launch / 1e3)
  print(json.dumps({
    'metric': 'mixed-shape group elements/s', 'value': n / (total / args.steps / 1e3), 'unit': 'elements/s',
    'n_gpus': 1, 'steps': args.steps, 'warmup': max(3, args.warmup), 'ms_per_step': total / args.steps,
    'higher_is_better': True, 'dtype': 'f32', 'data': 'synthetic',
    'config': {'workload': f'mixed-shape group: {b} basis functions, {q} quantities, FP32', 'elements': n,
               'plan': g.get_plan().key()},
    'accuracy': acc,
    'roofline': {'bound': 'fp32', 'achieved': flops / 1e12, 'peak': peak / 1e12, 'unit': 'TFLOP/s',
                 'frac': flops / peak, 'flops_per_element': nz, 'kernel': g.get_base_name(),
                 'peak_source': 'measured FP32 FFMA probe (libtfb200_runtime tfb_fma_peak_launch), same run'},
    'gpu_launches': args.steps, 'clocks': clocks.summary()}))


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--gpus', type=int, default=1)
  ap.add_argument('--steps', type=int, default=20)
  ap.add_argument('--warmup', type=int, default=5)
  ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
  ap.add_argument('--variant', default='auto')
  ap.add_argument('--elements', type=int, default=500000)
  ap.add_argument('--no-cpu', action='store_true')
  ap.add_argument('--no-extras', action='store_true')
  ap.add_argument('--workload', default='chain_o6', choices=['chain_o6', 'ew_update', 'mixed'],
                  help='chain_o6: the headline order-6 chain; ew_update: the elementwise stage alone; '
                       'mixed: one group of the mixed-shape workload (--basis, --quantities)')
  ap.add_argument('--basis', type=int, default=84)
  ap.add_argument('--quantities', type=int, default=27)
  args = ap.parse_args()
  if args.workload == 'ew_update':
    impl_elementwise(args)
    return
  if args.workload == 'mixed':
    impl_mixed_group(args)
    return
  from tensorforge_b200.runtime import ranks
  rank, world, _ = ranks.env_rank()
  if args.impl == 'reference':
    impl_reference(args, rank, world)
    return
  import torch
  dist = ranks.init('nccl')
  if dist is None:
    torch.cuda.set_device(0)
  try:
    impl_ours(args, rank, world, dist)
  finally:
    if dist is not None:
      dist.destroy_process_group()


if __name__ == '__main__':
  main()
