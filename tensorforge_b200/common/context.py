"""Generation context: target architecture, precision and options.

Same constructor and accessors as tensorforge/common/context.py:6-54, restricted to
NVIDIA B200 (`sm_100`, `sm_100a`) and the `cuda` backend. `Options` gains the knobs of
this generator: the arithmetic form of dense stages (`precision`) and how the tiling
variant is chosen (`tuner`).
"""
from math import ceil
from .basic_types import FloatingPointType

SUPPORTED_ARCHS = ('sm_100', 'sm_100a')
SUPPORTED_BACKENDS = ('cuda',)
PRECISIONS = ('plain', 'tf32x3', 'bf16x3', 'dmma')
TUNERS = ('heuristic', 'exhaustive', 'model')


class HwDescription:
  """Hardware record for B200 (one sm_100a GPU)."""

  def __init__(self, arch: str, backend: str):
    self.vec_unit_length = 32
    self.hw_fp_word_size = 4
    self.mem_access_align_size = 32
    self.max_local_mem_size_per_block = 227 * 1024
    self.max_threads_per_block = 1024
    self.max_reg_per_block = 64 * 1024
    self.max_threads_per_sm = 2048
    self.max_block_per_sm = 32
    self.manufacturer = 'nvidia'
    self.shmem_banks = 32
    self.num_sms = 148
    self.smem_per_sm = 228 * 1024
    self.tmem_columns = 512
    self.model = arch
    self.backend = backend


class VM:
  def __init__(self, hw_descr: HwDescription, fp_type: str):
    if fp_type not in ('float', 'double'):
      raise RuntimeError(f'unknown fp_type. Allowed float, double, given {fp_type}')
    self._hw_descr = hw_descr
    self._fp_type = fp_type
    self._real_literal = 'f' if fp_type == 'float' else ''

  def get_hw_descr(self):
    return self._hw_descr

  def get_real_literal(self):
    return self._real_literal

  def fp_as_str(self):
    return self._fp_type

  def bytes_per_real(self):
    return {'double': 8, 'float': 4}[self._fp_type]

  def align(self, num):
    v = self._hw_descr.vec_unit_length
    return ceil(num / v) * v

  def get_headers(self):
    return ['tensorforge_aux.h']


def vm_factory(arch: str, backend: str, fp_type: str):
  if backend not in SUPPORTED_BACKENDS or arch not in SUPPORTED_ARCHS:
    raise ValueError(f'Unknown gpu architecture: {backend} {arch}')
  return VM(HwDescription(arch, backend), fp_type)


class Options:
  def __init__(self,
               exact_contraction_length=False,
               align_shr_mem=True,
               enable_sync_block_opt=True,
               precision='plain',
               tuner='heuristic',
               variant=None):
    if precision not in PRECISIONS:
      raise ValueError(f'precision must be one of {PRECISIONS}, given {precision}')
    if tuner not in TUNERS:
      raise ValueError(f'tuner must be one of {TUNERS}, given {tuner}')
    self.exact_contraction_length: bool = exact_contraction_length
    self.align_shr_mem: bool = align_shr_mem
    self.enable_sync_block_opt = enable_sync_block_opt
    self.precision = precision
    self.tuner = tuner
    self.variant = variant


class Context:
  def __init__(self, arch: str, backend: str, fp_type: FloatingPointType, options: Options = None):
    self._vm = vm_factory(arch, backend, FloatingPointType.as_str(fp_type))
    self.fp_type = fp_type
    self._options = options if options is not None else Options()
    self.arch = arch
    self.backend = backend

  def set_fp_type(self, fp_type: FloatingPointType):
    self.fp_type = fp_type

  def fp_as_str(self):
    return FloatingPointType.as_str(self.fp_type)

  def get_vm(self):
    return self._vm

  def get_user_options(self):
    return self._options

  def align(self, num):
    hw = self._vm.get_hw_descr()
    align_length = (hw.vec_unit_length * hw.hw_fp_word_size) / self.fp_type.size()
    return int(ceil(num / align_length) * align_length)

  def align_range(self, begin, end):
    assert end > begin
    factor = self._vm.get_hw_descr().mem_access_align_size / self.fp_type.size()
    aligned_begin = begin - begin % factor
    aligned_end = end + (factor - end % factor) % factor
    return int(aligned_begin), int(aligned_end)
