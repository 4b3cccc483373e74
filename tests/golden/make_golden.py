"""Generate the golden vectors in this folder from the reference's own kernels.

Run from the repository root where the reference source tree is available:

    python tests/golden/make_golden.py            # all cases
    TFB_REFERENCE_ROOT=/path/to/reference python tests/golden/make_golden.py

For every case in oracle/cases.py this builds the reference generator's OpenMP output
(oracle/ref_omp.py), runs it on seeded inputs laid out as the launcher ABI expects
(oracle/harness.py) and stores inputs, outputs and the reference's kernel name in
`<case>_<fp>.npz`. Cases the reference cannot generate are recorded in
`reference_failures.txt` with the error it raised.
"""
import json
import os
import sys
import traceback

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import cases, harness, ref_omp  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
FP64_CASES = ('c0_gemm_ptr', 'chain_o6', 'three_matrices', 'sparse_a_batched')


def make(name, fp):
  dtype = np.float32 if fp == 'float' else np.float64
  builder = lambda ns: cases.build(name, ns)  # noqa: E731
  tag = f'golden_{name}_{fp}'
  ref_omp.build(tag, builder, fp)
  rk = ref_omp.RefKernel(tag)
  descrs = builder(cases.ns_from_module('tensorforge_b200'))
  n = cases.num_elements(name)
  layouts, mem = harness.make_memory(descrs, n, seed=1, dtype=dtype)
  inputs = {k: v.astype(dtype) for k, v in mem.buffers.items()}
  outputs = {k: v.copy() for k, v in inputs.items()}
  rk.run(layouts, outputs, n, scalars=mem.scalars)
  payload = {'n': np.int64(n)}
  meta = {'case': name, 'fp': fp, 'reference_kernel': rk.base_name, 'header': rk.header.strip(),
          'symbols': []}
  for lay in layouts:
    meta['symbols'].append({'name': lay.name, 'kind': lay.kind, 'extra_offset': int(lay.extra_offset),
                            'slot': int(lay.slot), 'size': int(lay.size)})
    if lay.kind == 'scalar':
      payload[f'scalar_{lay.name}'] = np.float64(mem.scalars[lay.name])
      continue
    payload[f'in_{lay.name}'] = inputs[lay.name]
    payload[f'out_{lay.name}'] = outputs[lay.name]
    if lay.starts is not None:
      payload[f'starts_{lay.name}'] = lay.starts
  payload['meta'] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
  np.savez_compressed(os.path.join(OUT, f'{name}_{fp}.npz'), **payload)


def main():
  failures = []
  names = sys.argv[1:] or list(cases.CASES)
  for name in names:
    for fp in ('float', 'double') if name in FP64_CASES else ('float',):
      try:
        make(name, fp)
        print('ok', name, fp)
      except Exception as e:  # the reference itself failed to generate this chain
        tb = traceback.format_exception_only(type(e), e)[-1].strip()
        failures.append(f'{name} {fp}: {tb}')
        print('reference failed', name, fp, tb)
  if not sys.argv[1:]:
    with open(os.path.join(OUT, 'reference_failures.txt'), 'w') as f:
      f.write('\n'.join(failures) + ('\n' if failures else ''))


if __name__ == '__main__':
  main()
