"""`import tensorforge` through tensorforge_b200/compat: scripts written against the
reference's module paths run unchanged on tensorforge_b200 (no GPU)."""
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COMPAT = os.path.join(REPO, 'tensorforge_b200', 'compat')

# the reference's example/gemm.py flow, written out: GemmDescr with alpha and beta on strided
# 56x18 x 18x18 operands, generated for sm_100a
SCRIPT = r'''
from tensorforge.common.context import Context
from tensorforge.generators.descriptions import GemmDescr
from tensorforge.common.basic_types import FloatingPointType, Addressing
from tensorforge.generators.generator import Generator
from tensorforge.common.matrix.boundingbox import BoundingBox
from tensorforge.common.matrix.tensor import Tensor, SubTensor
import tensorforge
a = SubTensor(Tensor([56, 18], Addressing.STRIDED, BoundingBox([0, 0], [56, 18])), BoundingBox([0, 0], [56, 18]))
b = SubTensor(Tensor([18, 18], Addressing.STRIDED, BoundingBox([0, 0], [18, 18])), BoundingBox([0, 0], [18, 18]))
c = SubTensor(Tensor([56, 18], Addressing.STRIDED, BoundingBox([0, 0], [56, 18])), BoundingBox([0, 0], [56, 18]))
gen = Generator([GemmDescr(trans_a=False, trans_b=False, a=a, b=b, c=c, alpha=1.1, beta=1.1)],
                Context(arch='sm_100a', backend='cuda', fp_type=FloatingPointType.FLOAT))
gen.generate()
assert type(gen).__module__ == 'tensorforge_b200.generators.generator'
assert tensorforge.get_routine_generator(None).__module__ == 'tensorforge_b200.frontend.yateto'
print(gen.get_header().strip())
'''


def test_reference_module_paths_resolve_to_tensorforge_b200():
  env = dict(os.environ, PYTHONPATH=os.pathsep.join([COMPAT, REPO]))
  r = subprocess.run([sys.executable, '-c', SCRIPT], env=env, capture_output=True, text=True, timeout=300)
  assert r.returncode == 0, r.stderr[-2000:]
  assert r.stdout.startswith('void launcher_kernel_')


def test_reference_example_imports_resolve():
  """Every name the reference's example scripts import from `tensorforge`."""
  env = dict(os.environ, PYTHONPATH=os.pathsep.join([COMPAT, REPO]))
  code = '\n'.join([
    'from tensorforge.common.aux import generate_tmp_matrix',
    'from tensorforge.common.basic_types import FloatingPointType, Addressing',
    'from tensorforge.common.context import Context',
    'from tensorforge.common.exceptions import GenerationError',
    'from tensorforge.common.matrix.boundingbox import BoundingBox',
    'from tensorforge.common.matrix.tensor import Tensor, SubTensor',
    'from tensorforge.generators.descriptions import GemmDescr, MultilinearDescr, FloatingPointType, Addressing',
    'from tensorforge.generators.generator import Generator',
    'from tensorforge.common.vm.vm import vm_factory',
    'from tensorforge.common.vm import vm; assert vm.vm_factory is vm_factory',
    'from tensorforge.generators.optree import Assignment',
    'from tensorforge import get_routine_generator, get_cmake_path, print_cmake_path, use_fusedgemm_cost',
    'import tensorforge.functions as f; f.tensor; f.scalar; f.assign',
    'print("ok")'])
  r = subprocess.run([sys.executable, '-c', code], env=env, capture_output=True, text=True, timeout=300)
  assert r.returncode == 0 and r.stdout.strip() == 'ok', r.stderr[-2000:]


def test_same_objects_under_both_names():
  env = dict(os.environ, PYTHONPATH=os.pathsep.join([COMPAT, REPO]))
  code = ('import tensorforge.generators.descriptions as a, tensorforge_b200.generators.descriptions as b; '
          'import tensorforge.common.matrix.tensor as t, tensorforge_b200.common.matrix.tensor as u; '
          'assert a is b and a.GemmDescr is b.GemmDescr and t.Tensor is u.Tensor; print("ok")')
  r = subprocess.run([sys.executable, '-c', code], env=env, capture_output=True, text=True, timeout=300)
  assert r.returncode == 0 and r.stdout.strip() == 'ok', r.stderr[-2000:]
