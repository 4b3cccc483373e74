"""CPU baseline: the reference's own OpenMP-backend kernels for the benchmark workloads.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). `build_all()` needs the reference
source tree (it runs the reference generator); the built libraries in oracle/_ref/ are
then used without it.
"""
import os

from . import cases, ref_omp

BENCH_CASES = {
  # tag: (case builder name, kwargs, fp)
  'bench_chain_o6_float': ('chain_o6', 'float'),
  'bench_chain_o6_double': ('chain_o6', 'double'),
  'bench_c0_gemm_ptr_float': ('c0_gemm_ptr', 'float'),
}


def build_all():
  for tag, (case, fp) in BENCH_CASES.items():
    ref_omp.build(tag, lambda ns, c=case: cases.build(c, ns), fp, opt='-O3')


def available(tag):
  return os.path.exists(os.path.join(ref_omp.REF_OUT, f'{tag}.so'))
