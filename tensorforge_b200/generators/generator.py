"""The code generator: descriptor list -> sm_100a kernel + C-ABI launcher.

Public surface mirrors tensorforge/generators/generator.py:52-505 (`Generator` with
`register`, `generate`, `get_kernel`, `get_launcher`, `get_header`, `get_base_name`,
`set_kernel_name`, `default_generate_call_site`, `generate_call_site`,
`get_helper_headers`). Operand naming (m*, t*), the ABI parameter list and the md5
kernel name follow the reference exactly (generator.py:301-362, :384-436), so an
emitted launcher has the same name and signature as the reference's CUDA backend
output and links in its place. Underneath, the chain is lowered to the chain IR,
planned for B200 and emitted by the sm_100a code generators.
"""
import hashlib
from typing import List

from ..common.basic_types import Addressing, GeneralLexicon, DataFlowDirection
from ..common.context import Context
from ..common.exceptions import GenerationError
from ..ir.chain import lower
from .descriptions import OperationDescription, MultilinearDescr, ElementwiseDescr


class RegmaxBlockPolicy:
  """Kept for interface compatibility (generator.py:38-50); planning is done by tensorforge_b200.plan."""

  def __init__(self, context, global_mem, mem_size_per_mult, num_threads):
    self._context = context


class Generator:
  NAME_ENCODING_LENGTH = 10

  def __init__(self, gemm_list: List[OperationDescription], context: Context,
               thread_block_policy_type=RegmaxBlockPolicy):
    self.descr_list = list(gemm_list)
    self._context = context
    self._base_kernel_name = None
    self._kernel = None
    self._launcher = None
    self._header = None
    self._matrix_list = None
    self._tmp_list = None
    self._globals = []            # [(tensor, stype)] in m-order, stype in batch|scalar|data
    self._is_registered = False
    self._chain = None
    self._plan = None
    self._emitted = None
    for d in self.descr_list:
      if not isinstance(d, (MultilinearDescr, ElementwiseDescr)):
        raise GenerationError(f'unsupported operation description: {type(d).__name__}')
    self._check_consistency_with_user_options()
    self._name_operands(self.descr_list)

  # ------------------------------------------------------------------ naming / ABI
  def set_kernel_name(self, name):
    self._base_kernel_name = name

  def register(self):
    self._collect_tmp_matrices()
    self._populate_global_scope()
    if not self._base_kernel_name:
      self._generate_kernel_name()
    self._is_registered = True

  def _check_consistency_with_user_options(self):
    opts = self._context.get_user_options()
    for d in self.descr_list:
      if d.is_strict_match() != opts.exact_contraction_length:
        raise RuntimeError('gemm list is not consistent with user options. '
                           f'`strict_math` in gemm descr. set to {d.is_strict_match()}, '
                           f'but `exact_contraction_length` is set to {opts.exact_contraction_length}')

  def _name_operands(self, descr_list):
    seen = {}
    for d in descr_list:
      for sub in d.matrix_list():
        seen.setdefault(id(sub.tensor), sub.tensor)
    self._matrix_list = list(seen.values())
    tmp_counter = op_counter = 0
    for t in self._matrix_list:
      if t.is_tmp:
        t.name = f't{tmp_counter}'
        tmp_counter += 1
      else:
        t.name = f'm{op_counter}'
        op_counter += 1

  def _collect_tmp_matrices(self):
    self._tmp_list = [t for t in self._matrix_list if t.is_tmp]

  def _populate_global_scope(self):
    self._globals = []
    for t in self._matrix_list:
      if t.is_tmp:
        continue
      if t.has_values() and len(t.get_values()) < 16:
        stype = 'data'
      elif t.addressing == Addressing.SCALAR:
        stype = 'scalar'
      else:
        stype = 'batch'
      self._globals.append((t, stype))

  def _generate_kernel_name(self):
    long_name = [t.gen_descr() for t, _ in self._globals]
    long_name.extend(str(d) for d in self.descr_list)
    md5 = hashlib.md5(', '.join(long_name).encode()).hexdigest()
    self._base_kernel_name = f'kernel_{md5[:Generator.NAME_ENCODING_LENGTH]}'

  def get_base_name(self):
    return self._base_kernel_name

  def _datatype(self, t):
    return self._context.fp_as_str() if t.datatype is None else str(t.datatype)

  def _generate_base_params_list(self, with_types=True, with_defaults=False, alias=False):
    params = []
    for t, _ in self._globals:
      name = (t.alias if alias and t.alias else t.name)
      dt = self._datatype(t)
      if t.addressing == Addressing.SCALAR:
        params.append(f'{dt} {name}' if with_types else f'{name}')
      else:
        const = 'const ' if t.direction == DataFlowDirection.SOURCE else ''
        btype = f'{const}{dt}{t.addressing.to_pointer()}' if with_types else ''
        params.append(f'{btype} {name}')
        if t.addressing != Addressing.NONE:
          otype = 'unsigned' if with_types else ''
          params.append(f'{otype} {name}{GeneralLexicon.EXTRA_OFFSET}')
    params.append(f'{"size_t" if with_types else ""} {GeneralLexicon.NUM_ELEMENTS}')
    params.append(f'{"unsigned*" if with_types else ""} {GeneralLexicon.FLAGS_NAME} '
                  f'{"= nullptr" if with_defaults else ""}')
    return params

  def _generate_launcher_proto(self, with_defaults=True):
    params = self._generate_base_params_list(with_types=True, with_defaults=with_defaults)
    params.append(f'void* {GeneralLexicon.STREAM_PTR_STR}{" = nullptr" if with_defaults else ""}')
    return f'void launcher_{self._base_kernel_name}({", ".join(params)})'

  def _status_entry(self):
    """`extern "C" int tfb_launch_<name>(...)`: the launcher's parameters (no defaults),
    returning the CUDA status of the launch (0 = success) for FFI callers that bind a
    return code (ctypes, cgo). Emitted after the launcher; the launcher itself keeps the
    reference's `void` signature and leaves the status for tensorforge_last_status()."""
    proto = self._generate_launcher_proto(with_defaults=False)
    args = [a.strip() for a in self._generate_base_params_list(with_types=False)]
    args.append(GeneralLexicon.STREAM_PTR_STR)
    return (f'\n\nextern "C" int tfb_launch_{self._base_kernel_name}{proto[proto.index("("):]} {{\n'
            f'  (void)tensorforge_last_status();\n'
            f'  launcher_{self._base_kernel_name}({", ".join(args)});\n'
            f'  return tensorforge_last_status();\n}}')

  def abi_params(self):
    """[(c type, name)] of the launcher in order (used by the ctypes binding)."""
    out = []
    for t, _ in self._globals:
      dt = self._datatype(t)
      if t.addressing == Addressing.SCALAR:
        out.append((dt, t.name))
      else:
        const = 'const ' if t.direction == DataFlowDirection.SOURCE else ''
        out.append((f'{const}{dt}{t.addressing.to_pointer()}', t.name))
        if t.addressing != Addressing.NONE:
          out.append(('unsigned', f'{t.name}{GeneralLexicon.EXTRA_OFFSET}'))
    out += [('size_t', 'numElements'), ('unsigned*', 'flags'), ('void*', 'streamPtr')]
    return out

  def abi_symbols(self):
    """[(tensor, stype)] of the ABI symbols in m-order."""
    return list(self._globals)

  def default_generate_call_site(self):
    if not self._is_registered:
      raise RuntimeError('generator is not registered. Call register first.')
    args = self._generate_base_params_list(with_types=False, alias=True)
    args.append(GeneralLexicon.FLAGS_NAME)
    args.append(GeneralLexicon.STREAM_PTR_STR)
    return f'launcher_{self._base_kernel_name}({", ".join(args)});'

  def generate_call_site(self, mat_name_map, offset_name_map, num_element, flags=None, stream=None):
    args = []
    for t, _ in self._globals:
      if t.alias in mat_name_map:
        args.append(mat_name_map[t.alias])
        if t.addressing not in (Addressing.SCALAR, Addressing.NONE):
          args.append(offset_name_map[t.alias])
    args.append(num_element)
    if flags:
      args.append(flags)
    if stream:
      args.append(stream)
    return f'launcher_{self._base_kernel_name}({", ".join(args)});'

  def get_helper_headers(self):
    return ['tensorforge_aux.h']

  # ------------------------------------------------------------------ generation
  def generate(self):
    if not self._is_registered:
      self.register()
    from ..plan import make_plan
    from ..codegen import emit
    self._chain = lower(self.descr_list, self._matrix_list, self._globals, self._context.fp_type)
    self._plan = make_plan(self._chain, self._context, self._tuned_variant())
    self._emitted = emit(self._chain, self._plan, self._context, self._base_kernel_name,
                         self._generate_launcher_proto(with_defaults=False), self._globals)
    self._emitted.launcher += self._status_entry()
    self._kernel = self._emitted.kernel
    self._launcher = self._emitted.launcher
    self._header = f'{self._generate_launcher_proto(with_defaults=True)};\n'

  def _tuned_variant(self):
    """Variant picked by Options.tuner ('model' / 'exhaustive'), None for the planner's own.

    Chains without an explicit variant are tuned: plain-precision ones by either tuner
    (the cost model was trained on FP32 timings, so FP64 chains keep the planner's choice
    under 'model'), TF32x3 ones by the exhaustive tuner over the tensor-core variants.
    """
    opts = self._context.get_user_options()
    if opts.tuner == 'heuristic' or opts.variant:
      return None
    if opts.precision != 'plain' and not (opts.tuner == 'exhaustive' and opts.precision == 'tf32x3'):
      return None
    from ..tune import select
    if opts.tuner == 'model':
      if self._context.fp_type.size() != 4:
        return None
      return select.model_choice(self._chain, 4)
    return select.exhaustive_choice(self.descr_list, self._context)

  def get_kernel(self):
    return self._kernel

  def get_launcher(self):
    return self._launcher

  def get_header(self):
    return self._header

  def get_status_header(self):
    """Declaration of the status-returning twin of the launcher (`tfb_launch_<name>`,
    emitted after the launcher by `get_launcher()`); `get_header()` stays the reference's
    single prototype."""
    proto = self._generate_launcher_proto(with_defaults=True)
    return f'extern "C" int tfb_launch_{self._base_kernel_name}{proto[proto.index("("):]};\n'

  # ------------------------------------------------------------------ additions
  def get_source(self):
    """A complete .cu translation unit (includes + kernel + launcher)."""
    return self._emitted.source()

  def get_plan(self):
    return self._plan

  def get_chain(self):
    return self._chain

  def get_context(self):
    return self._context
