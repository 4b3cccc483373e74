"""Frontend and launcher ABI: identical names and signatures to the reference's CUDA backend."""
import pytest

from oracle import cases
from tensorforge_b200.common.basic_types import FloatingPointType, Addressing
from tensorforge_b200.common.context import Context, Options
from tensorforge_b200.common.exceptions import GenerationError
from tensorforge_b200.common.matrix.tensor import Tensor, SubTensor
from tensorforge_b200.common.matrix.boundingbox import BoundingBox
from tensorforge_b200.generators.generator import Generator
from tensorforge_b200.generators.descriptions import GemmDescr
from tests.golden_io import golden_files, golden_ids, load


def _gen(case, fp='float'):
  ns = cases.ns_from_module('tensorforge_b200')
  ftype = FloatingPointType.FLOAT if fp == 'float' else FloatingPointType.DOUBLE
  g = Generator(cases.build(case, ns), Context('sm_100a', 'cuda', ftype))
  g.register()
  return g


@pytest.mark.parametrize('path', golden_files(), ids=golden_ids())
def test_kernel_name_and_prototype_match_reference(path):
  z, meta = load(path)
  g = _gen(meta['case'], meta['fp'])
  assert g.get_base_name() == meta['reference_kernel']
  proto = g._generate_launcher_proto(with_defaults=True) + ';'
  assert proto == meta['header']


def test_header_has_reference_linkage_and_defaults():
  """The launcher keeps the reference's C++ linkage (generator.py:198-199, :426-436);
  the status-returning twin has C linkage for FFI callers."""
  g = _gen('c0_gemm_ptr')
  g.generate()
  h = g.get_header()
  assert h.startswith('void launcher_kernel_')
  assert 'unsigned* flags = nullptr, void* streamPtr = nullptr);' in h
  launcher = g.get_launcher()
  assert launcher.count(f'void launcher_{g.get_base_name()}(') == 1
  assert 'extern "C" void launcher_' not in launcher
  # the status-returning entry point follows the launcher, same parameters without defaults
  params = g._generate_launcher_proto(with_defaults=False).split('(', 1)[1]
  assert f'extern "C" int tfb_launch_{g.get_base_name()}({params} {{' in launcher
  assert 'nullptr' not in launcher.split('tfb_launch_')[1].split('{')[0]
  assert g.get_status_header() == 'extern "C" ' + h.replace('void launcher_', 'int tfb_launch_')


def test_call_sites():
  g = _gen('c0_gemm_ptr')
  assert g.default_generate_call_site().startswith(f'launcher_{g.get_base_name()}(')
  for t, _ in g.abi_symbols():
    t.alias = t.name.upper()
  cs = g.generate_call_site({'M0': 'c', 'M1': 'a', 'M2': 'b'}, {'M0': 'oc', 'M2': 'ob'}, 'n', 'fl', 'st')
  assert cs == f'launcher_{g.get_base_name()}(c, oc, a, b, ob, n, fl, st);'


def test_context_rejects_other_targets():
  with pytest.raises(ValueError):
    Context('sm_90', 'cuda', FloatingPointType.FLOAT)
  with pytest.raises(ValueError):
    Context('sm_100', 'hip', FloatingPointType.FLOAT)
  with pytest.raises(ValueError):
    Options(precision='int8')
  Context('sm_100', 'cuda', FloatingPointType.DOUBLE)


def test_bbox_validation():
  with pytest.raises(GenerationError):
    Tensor([4, 4], Addressing.STRIDED, BoundingBox([0, 0], [5, 4]))


def test_writing_shared_operand_rejected():
  A = Tensor([4, 4], Addressing.NONE)
  B = Tensor([4, 4], Addressing.NONE)
  C = Tensor([4, 4], Addressing.NONE)
  g = Generator([GemmDescr(False, False, SubTensor(A), SubTensor(B), SubTensor(C))],
                Context('sm_100', 'cuda', FloatingPointType.FLOAT))
  with pytest.raises(GenerationError):
    g.generate()


def test_every_case_generates():
  for name in cases.CASES:
    g = _gen(name)
    g.generate()
    src = g.get_source()
    assert f'launcher_{g.get_base_name()}' in src
