"""CPU baseline: the reference's own OpenMP-backend kernels for the benchmark workloads.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). `build_all()` needs the reference
source tree (it runs the reference generator); the built libraries in oracle/_ref/ are
then used without it.
"""
import os

from . import cases, ref_omp

BENCH_CASES = {
  # tag: (case name, fp)
  'bench_chain_o6_float': ('chain_o6', 'float'),
  'bench_chain_o6_double': ('chain_o6', 'double'),
  'bench_c0_gemm_ptr_float': ('c0_gemm_ptr', 'float'),
}
# one reference kernel per group of the mixed-shape workload (basis x quantities)
for _b in cases.MIXED_BASES:
  for _q in cases.MIXED_QUANTITIES:
    BENCH_CASES[f'bench_mixed_{_b}_{_q}_float'] = (f'mixed_{_b}_{_q}', 'float')


def mixed_tag(basis, quantities):
  return f'bench_mixed_{basis}_{quantities}_float'


def build_all(jobs=8):
  """Build every benchmark case's reference kernel (g++ runs in parallel; the large-basis
  chains take minutes each)."""
  from concurrent.futures import ThreadPoolExecutor
  todo = [(tag, case, fp) for tag, (case, fp) in BENCH_CASES.items() if not available(tag)]
  for tag, case, fp in todo:  # generation (Python) serially, compilation in parallel
    ref_omp.generate_source(tag, lambda ns, c=case: cases.build(c, ns), fp)
  with ThreadPoolExecutor(max_workers=jobs) as pool:
    list(pool.map(lambda t: ref_omp.compile_source(t[0], opt='-O3'), todo))


def available(tag):
  return all(os.path.exists(os.path.join(ref_omp.REF_OUT, f'{tag}.{ext}')) for ext in ('so', 'meta'))
