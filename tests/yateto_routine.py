"""Shared by the yateto routine tests: a chain generated through the yateto gateway with mock
yateto objects, written to a routine file, and a driver that calls the launcher through the
gateway's own call site, the way yateto's generated kernel::execute() does."""
from tests.test_yateto_frontend import YTensor, CSCMemoryLayout, Arch, Cpp, Cache


def generate_routine(tmp_path):
  from tensorforge_b200 import interop
  from tensorforge_b200.common.basic_types import Addressing
  FE = interop.get_routine_generator(None)
  fe = FE(Arch())
  K = YTensor('kDivM', (56, 56), const=True,
              layout=CSCMemoryLayout((56, 56), [(i, j) for j in range(56) for i in range(56) if (i * 7 + j) % 3]))
  Q = YTensor('Q', (56, 9))
  S = YTensor('star', (9, 9))
  T = YTensor('_tmp0', (56, 9), tmp=True)
  out = YTensor('Qout', (56, 9))
  fe.add_linear_operation(T, [K, Q], [[0, -1], [-1, 1]], [[0, 1], [0, 1]], False)
  fe.add_linear_operation(out, [T, S], [[0, -1], [-1, 1]], [[0, 1], [0, 1]], False)
  cpp, cache = Cpp(), Cache()
  g = fe.generate(cpp, cache)
  writer = cache.routines[g.get_base_name()]
  path = tmp_path / 'subroutine.cu'
  writer('r', str(path))
  inc = Cpp()
  writer.header(inc)
  params = []
  for t, _ in g.abi_symbols():
    a = t.alias
    if t.addressing == Addressing.NONE:
      params.append(f'float* {a}')
    elif t.addressing == Addressing.PTR_BASED:
      params += [f'float** {a}', f'unsigned extraOffset_{a}']
    else:
      params += [f'float* {a}', f'unsigned extraOffset_{a}']
  params += ['size_t numElements', 'unsigned* flags', 'void* streamPtr']
  source = (''.join(f'#include <{h}>\n' if not h.endswith('.h') or h.startswith('cuda') else f'#include "{h}"\n'
                    for h in inc.included)
            + path.read_text()
            + f'\nextern "C" void yateto_execute({", ".join(params)}) {{\n  {cpp.lines[0]}\n}}\n')
  return g, fe.generator._descr_list, source
