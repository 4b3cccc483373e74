"""GPU: tcgen05 split-precision chains vs the FP64 oracle and the plain FP32 path.

Tolerances (relative L2 over the whole output, the reference test suite's norm):
TF32x3 <= 1e-6 (the order-6 target), BF16x3 <= 5e-5 (16 significant bits per product).
"""
import ctypes

import numpy as np
import pytest

from oracle import cases, harness, multilinear

pytestmark = pytest.mark.gpu

TOL = {'tf32x3': 1e-6, 'bf16x3': 5e-5}


def _run(case, precision, n, seed=3, dist='uniform', use_flags=False, variant=None):
  import torch
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  g = make(case, 'float', precision=precision, **({'variant': variant} if variant else {}))
  assert g.get_plan().strategy == 'tcsplit', g.get_plan()
  k = compile_generator(g)
  descrs = cases.build(case, cases.ns_from_module('tensorforge_b200'))
  lay, mem = harness.make_memory(descrs, n, seed=seed, dist=dist)
  flags = harness.make_flags(n, seed) if use_flags else None
  dev, kw, keep = {}, {'numElements': n}, []
  for l in lay:
    if l.kind == 'scalar':
      kw[l.name] = float(mem.scalars[l.name])
      continue
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
    elif l.kind == 'ptr':  # device array of element pointers (without the extra offset)
      starts = np.asarray(l.starts, dtype=np.int64) - l.extra_offset
      ptrs = torch.tensor(dev[l.name].data_ptr() + starts * 4, dtype=torch.int64, device='cuda')
      keep.append(ptrs)
      kw[l.name] = ptrs
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  if flags is not None:
    kw['flags'] = torch.tensor(flags, dtype=torch.int32, device='cuda')
  k(**kw)
  torch.cuda.synchronize()
  lib = ctypes.CDLL(k.so_path)
  errf = getattr(lib, f'tfb_kernel_error_{g.get_base_name()}')
  errf.argtypes = [ctypes.c_void_p]
  assert errf(None) == 0
  # oracle on float32-exact inputs
  multilinear.evaluate(descrs, mem, n, flags=flags)
  out = [l for l in lay if l.kind in ('strided', 'ptr') and l.tensor.direction.name != 'SOURCE'][0]
  got = dev[out.name].double().cpu().numpy()
  ref = mem.buffers[out.name]
  return got, ref, out, flags


@pytest.mark.parametrize('precision', ['tf32x3', 'bf16x3'])
@pytest.mark.parametrize('n', [1, 14, 333, 4099])
def test_chain_o6_split(precision, n):
  got, ref, out, _ = _run('chain_o6', precision, n)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= TOL[precision], rel


def test_chain_o6_flags_mask_elements():
  got, ref, out, flags = _run('chain_o6', 'tf32x3', 517, use_flags=True)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6
  # masked elements keep their previous contents exactly (the oracle leaves them untouched)
  for e in np.nonzero(flags == 0)[0][:5]:
    s = out.starts[e]
    assert np.array_equal(got[s:s + 504], ref[s:s + 504])


def test_chain_o6_loguniform_tf32x3():
  """Values with magnitudes spanning 1e-3..1e3 (precision-form inputs)."""
  got, ref, _, _ = _run('chain_o6', 'tf32x3', 777, dist='loguniform')
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


def test_other_shapes_split():
  got, ref, _, _ = _run('chain_o4_q27', 'tf32x3', 301)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


def _b_offset_seeds():
  """Seeds whose random extra offset leaves the per-element B operand (Q, 504 values) 16-byte
  aligned (staged with one bulk copy per tile) and misaligned (staged with cp.async)."""
  descrs = cases.build('chain_o6', cases.ns_from_module('tensorforge_b200'))
  found = {}
  for seed in range(64):
    lay = harness.make_layout(descrs, 8, seed)
    b = [l for l in lay if l.kind == 'strided' and l.tensor.direction.name == 'SOURCE' and l.slot == 504]
    found.setdefault(b[0].extra_offset % 4 == 0, seed)
    if len(found) == 2:
      return found[True], found[False]
  raise AssertionError('no seed covers both staging paths')


@pytest.mark.parametrize('aligned', [True, False])
def test_chain_o6_bulk_and_fallback_staging(aligned):
  seed = _b_offset_seeds()[0 if aligned else 1]
  got, ref, _, _ = _run('chain_o6', 'tf32x3', 2999, seed=seed)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


@pytest.mark.parametrize('n', [1, 29, 4099])
def test_chain_o6_one_pass_pipeline(n):
  """The one-pass producer pipeline without separate epilogue warps (plan option pipe=2,
  the form used where the warp-specialised pipeline does not apply)."""
  got, ref, _, _ = _run('chain_o6', 'tf32x3', n, variant={'pipe': 2})
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


PIPE3_OPTIONS = [{'form': 'u', 'qreg': 1}, {'form': 'u', 'slots': 2}, {'form': 'u', 'loader': 1},
                 {'form': 'u', 'urows': 2}, {'form': 'u', 'urows': 2, 'fuse': 1}, {'form': 'u', 'qreg': 1, 'fuse': 1},
                 {'form': 'u', 'urows': 2, 'loader': 2}, {'form': 'u', 'urows': 2, 'fuse': 1, 'loader': 2},
                 {'form': 'u', 'urows': 1, 'fuse': 0, 'loader': 0},
                 {'form': 'u', 'fuse': 0}, {'form': 'u', 'loader': 3}, {'form': 'u', 'sleep': 0},
                 {'form': 'u', 'sleep': 0, 'loader': 2}, {'form': 'u', 'ostage': 0},
                 {'form': 'u', 'opad': 1}, {'form': 'u', 'uwarp': 0},
                 {'form': 'u', 'direct': 1}, {'form': 'u', 'l64': 1},
                 {'form': 'u', 'oswz': 1}, {'form': 'u', 'estg': 1},
                 {'form': 'u', 'sleep': 1}, {'form': 'u', 'sleep': 2}, {'form': 'u', 'lpk': 0},
                 {'form': 'u', 'epk': 0}, {'form': 'u', 'sleep': 3}]


@pytest.mark.parametrize('variant', PIPE3_OPTIONS, ids=lambda v: ','.join(f'{k}={x}' for k, x in v.items() if k != 'form'))
@pytest.mark.parametrize('n', [1, 333, 4099])
def test_warp_specialised_pipeline_options(variant, n):
  """Options of the warp-specialised pipeline: B rows read into registers a tile ahead,
  two A slots with two accumulator pairs, a loader warp, two U rows per producer."""
  got, ref, _, _ = _run('chain_o6', 'tf32x3', n, variant=variant)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


@pytest.mark.parametrize('variant', PIPE3_OPTIONS[:2] + PIPE3_OPTIONS[4:], ids=lambda v: ','.join(f'{k}={x}' for k, x in v.items() if k != 'form'))
def test_warp_specialised_pipeline_options_flags_loguniform(variant):
  got, ref, out, flags = _run('chain_o6', 'tf32x3', 517, use_flags=True, variant=variant)
  assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6
  for e in np.nonzero(flags == 0)[0][:5]:
    st = out.starts[e]
    assert np.array_equal(got[st:st + 504], ref[st:st + 504])
  got, ref, _, _ = _run('chain_o6', 'tf32x3', 777, dist='loguniform', variant=variant)
  assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6


@pytest.mark.parametrize('direct', [0, 1])
@pytest.mark.parametrize('n', [1, 333, 2001])
def test_warp_specialised_pipeline_pointer_arrays(n, direct):
  """Q, S and out through device arrays of element pointers: the B blocks take the copy
  fallback (no contiguous tile), the output the per-lane stores; with the direct-lane
  producers the loader reads the S values through the pointer tables."""
  variant = {'form': 'u', 'direct': direct}
  g = __import__('tensorforge_b200.kernels', fromlist=['make']).make('chain_o6_ptr', 'float', precision='tf32x3',
                                                                     variant=variant)
  assert g.get_plan().params['pipe'] == 3
  assert int(g.get_plan().params.get('direct', 0)) == direct
  got, ref, _, _ = _run('chain_o6_ptr', 'tf32x3', n, variant=variant)
  assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6


@pytest.mark.parametrize('case,n', [('chain_o4_q27', 1), ('chain_o4_q27', 77), ('chain_o4_q27', 1001)])
def test_warp_specialised_pipeline_other_shape(case, n):
  """27 quantities: 4 elements per tile, 24-column A slots, 32-column accumulators."""
  g = __import__('tensorforge_b200.kernels', fromlist=['make']).make(case, 'float', precision='tf32x3')
  assert g.get_plan().params['pipe'] == 3
  got, ref, _, _ = _run(case, 'tf32x3', n)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


@pytest.mark.parametrize('precision', ['tf32x3', 'bf16x3'])
def test_chain_o6_per_term_pipeline(precision):
  """The per-term producer pipeline (plan option pipe=1), kept for shapes whose buffers
  for the one-pass pipeline do not fit in shared memory."""
  got, ref, _, _ = _run('chain_o6', precision, 1333, variant={'pipe': 1})
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= TOL[precision], rel


@pytest.mark.parametrize('case', ['c0_gemm_ptr', 'c0_gemm_strided', 'gemm_add', 'chain_o3_dense', 'sparse_a_shared'])
def test_other_chains_on_tensor_cores(case):
  """Pointer arrays (cp.async staging, per-lane output stores), accumulation into the
  output, a term without R, dense and sparse shared operands, all at TF32x3."""
  got, ref, _, _ = _run(case, 'tf32x3', 203)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


FORM_U = {'form': 'u'}
FORM_B = {'form': 'b'}


FORM_B_2ACC = {'form': 'b', 'acc': 2, 'bbuf': 2}
FORM_B_WS = {'form': 'b', 'ws': 1}


@pytest.mark.parametrize('form', [FORM_B, FORM_B_2ACC, FORM_B_WS, FORM_U],
                         ids=['formB', 'formB_2acc_2buf', 'formB_warp_specialized', 'formU'])
@pytest.mark.parametrize('n', [1, 7, 8, 333, 4099])
def test_chain_o6_both_operand_forms(form, n):
  """Operand form B (the per-element input as the MMA B operand, R applied in the epilogue)
  and form U (U = B R formed on CUDA cores, the MMA A operand in tensor memory)."""
  got, ref, _, _ = _run('chain_o6', 'tf32x3', n, variant=dict(form))
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


@pytest.mark.parametrize('form', [FORM_B, FORM_B_2ACC, FORM_B_WS, FORM_U], ids=['formB', 'formB_2acc_2buf', 'formB_ws', 'formU'])
@pytest.mark.parametrize('case', ['c0_gemm_ptr', 'c0_gemm_strided'])
def test_form_b_single_term(case, form):
  """One term (the A block stacked with itself, elements split between the lane halves),
  pointer-array and strided operands, no R."""
  from tensorforge_b200.kernels import make
  assert make(case, 'float', precision='tf32x3', variant=dict(form)).get_plan().params.get('form', 'u') == form['form']
  got, ref, _, _ = _run(case, 'tf32x3', 1001, variant=dict(form))
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel


@pytest.mark.parametrize('form', [FORM_B, FORM_B_WS], ids=['formB', 'formB_ws'])
def test_form_b_flags_and_loguniform(form):
  got, ref, out, flags = _run('chain_o6', 'tf32x3', 611, use_flags=True, variant=dict(form))
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= 1e-6, rel
  for e in np.nonzero(flags == 0)[0][:5]:
    s = out.starts[e]
    assert np.array_equal(got[s:s + 504], ref[s:s + 504])
  got, ref, _, _ = _run('chain_o6', 'tf32x3', 777, dist='loguniform', variant=dict(form))
  assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6


FORM_U_AHEAD = {'form': 'u', 'ahead': 1}


@pytest.mark.parametrize('n', [1, 13, 14, 15, 333, 4099])
def test_form_u_split_ahead(n):
  """Form U with the next term's column read and split while the previous term's tensor
  memory stores complete (plan option `ahead`): sizes around the 14-element tile, flags,
  log-uniform values."""
  from tensorforge_b200.kernels import make
  assert make('chain_o6', 'float', precision='tf32x3', variant=dict(FORM_U_AHEAD)).get_plan().params.get('ahead') == 1
  got, ref, _, _ = _run('chain_o6', 'tf32x3', n, variant=dict(FORM_U_AHEAD))
  assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6
  if n == 333:
    got, ref, out, flags = _run('chain_o6', 'tf32x3', 611, use_flags=True, variant=dict(FORM_U_AHEAD))
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6
    for e in np.nonzero(flags == 0)[0][:5]:
      s = out.starts[e]
      assert np.array_equal(got[s:s + 504], ref[s:s + 504])
    got, ref, _, _ = _run('chain_o6', 'tf32x3', 777, dist='loguniform', variant=dict(FORM_U_AHEAD))
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6


@pytest.mark.parametrize('probe', [{'wait_probe': 4096}, {'wait_probe_ns': 50000000}],
                         ids=['polls', 'global_timer'])
def test_bounded_wait_runs_out_and_context_stays_usable(probe):
  """Failure detection without a fault: a kernel built with a bounded wait on an mbarrier
  that nothing arrives on (plan option `wait_probe`: 4,096 polls of the spinning wait, or
  `wait_probe_ns`: 50 ms of the global timer in the sleeping wait; before any copy or MMA is
  issued) gives up, records error 30 in its error word and returns; the launch itself
  succeeds, the outputs are untouched, reading the error word clears it, and the regular
  kernel then runs in the same context and matches the oracle."""
  import time
  import torch
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  n = 333
  g = make('chain_o6', 'float', precision='tf32x3', variant=probe)
  key, val = next(iter(probe.items()))
  assert g.get_plan().params.get(key) == val
  k = compile_generator(g)
  descrs = cases.build('chain_o6', cases.ns_from_module('tensorforge_b200'))
  lay, mem = harness.make_memory(descrs, n, seed=5)
  dev, kw = {}, {'numElements': n}
  for l in lay:
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  out = [l for l in lay if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE'][0]
  before = dev[out.name].clone()
  torch.cuda.synchronize()
  t0 = time.time()
  k(**kw)
  torch.cuda.synchronize()
  if key == 'wait_probe_ns':
    # the sleeping wait gave up after its time limit, not earlier
    assert time.time() - t0 >= val * 1e-9
  errf = getattr(ctypes.CDLL(k.so_path), f'tfb_kernel_error_{g.get_base_name()}')
  errf.argtypes = [ctypes.c_void_p]
  assert errf(None) == 30
  assert errf(None) == 0  # read and cleared
  assert torch.equal(dev[out.name], before)
  got, ref, _, _ = _run('chain_o6', 'tf32x3', n, seed=5)
  assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6


@pytest.mark.parametrize('precision,variant', [('tf32x3', None), ('tf32x3', {'form': 'u', 'direct': 1}),
                                               ('tf32x3', {'pipe': 2}), (None, None)],
                         ids=['ws_pipeline', 'direct_lanes', 'one_pass', 'plain_fp32'])
def test_empty_batch_and_all_masked_elements(precision, variant):
  """Edge cases of the launcher contract: numElements = 0 launches nothing and returns 0;
  with every flag 0 the kernel runs over all tiles and writes no output value. In both the
  outputs keep their previous contents bit for bit and the error word stays 0."""
  import torch
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  kw_make = {}
  if precision:
    kw_make['precision'] = precision
  if variant:
    kw_make['variant'] = variant
  g = make('chain_o6', 'float', **kw_make)
  k = compile_generator(g)
  n = 333
  descrs = cases.build('chain_o6', cases.ns_from_module('tensorforge_b200'))
  lay, mem = harness.make_memory(descrs, n, seed=9)
  dev, kw = {}, {'numElements': n}
  for l in lay:
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  out = [l for l in lay if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE'][0]
  before = dev[out.name].clone()
  k(**dict(kw, numElements=0))
  torch.cuda.synchronize()
  assert torch.equal(dev[out.name], before)
  kw['flags'] = torch.zeros(n, dtype=torch.int32, device='cuda')
  k(**kw)
  torch.cuda.synchronize()
  assert torch.equal(dev[out.name], before)
  errf = getattr(ctypes.CDLL(k.so_path), f'tfb_kernel_error_{g.get_base_name()}', None)
  if errf is not None:
    errf.argtypes = [ctypes.c_void_p]
    assert errf(None) == 0
