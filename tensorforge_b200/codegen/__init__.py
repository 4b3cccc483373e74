"""sm_100a code generators and the launcher emitter.

`emit` turns a planned chain into the kernel text and a launcher whose name, parameter
list and C++ linkage are the reference CUDA backend's (tensorforge/generators/generator.py:
164-196, :426-436), so object code compiled against the reference's declaration links
unchanged. C, ctypes and other FFI callers bind `tfb_launch_<name>` instead (emitted by
the generator after the launcher, `extern "C"`, same parameters, returning the status).
Launcher behaviour kept from the reference: `streamPtr` is a `cudaStream_t` (nullptr ->
default stream), the launch is asynchronous, the caller owns every buffer and pointer
array and the launcher allocates nothing, and errors go through `CHECK_ERR`.
Additions: `numElements == 0` returns without a launch, the dynamic shared-memory
attribute is set once per device in a thread-safe way, and each error is also kept as
a status code readable through `tensorforge_last_status()`.
"""
from dataclasses import dataclass

from .generic import emit_generic

PRELUDE = '''#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <atomic>
#include <mutex>
#include <cstdio>
#include "tensorforge_aux.h"
'''


@dataclass
class Emitted:
  kernel: str
  launcher: str
  extra_prelude: str = ''

  def source(self):
    return PRELUDE + self.extra_prelude + '\n' + self.kernel + '\n\n' + self.launcher + '\n'


def emit_launcher(proto, launch):
  """Launcher body for a kernel described by `launch` (kernel, block, elements_per_block, smem, args)."""
  kname = launch['kernel']
  epb = launch['elements_per_block']
  smem = launch['smem']
  grid_expr = launch.get('grid', f'(numElements + {epb} - 1) / {epb}')
  pre = launch.get('pre', '')
  lines = [f'{proto} {{']
  lines.append('  if (numElements == 0) return;')
  lines.append(f'  const size_t blocks = {grid_expr};')
  lines.append(f'  dim3 block({launch["block"]}, 1, 1);')
  lines.append('  dim3 grid((unsigned)(blocks < 2147483647u ? blocks : 2147483647u), 1, 1);')
  lines.append('  int device = 0;')
  lines.append('  cudaGetDevice(&device);')
  lines.append('  static std::atomic<int> smemSet[64];')
  lines.append(f'  if (device < 64 && smemSet[device].load(std::memory_order_acquire) == 0) {{')
  lines.append(f'    cudaFuncSetAttribute({kname}, cudaFuncAttributeMaxDynamicSharedMemorySize, {smem});')
  lines.append('    CHECK_ERR;')
  lines.append('    smemSet[device].store(1, std::memory_order_release);')
  lines.append('  }')
  lines.append('  cudaStream_t stream = (streamPtr != nullptr) ? static_cast<cudaStream_t>(streamPtr) : 0;')
  if pre:
    lines.append(pre)
  if not launch.get('launched'):  # else `pre` launched the kernel itself
    lines.append(f'  {kname}<<<grid, block, {smem}, stream>>>({", ".join(launch["args"])});')
    lines.append('  CHECK_ERR;')
  lines.append('}')
  return '\n'.join(lines)


def emit(chain, plan, context, base_name, proto, globals_):
  if plan.strategy == 'generic':
    kernel, launch = emit_generic(chain, plan, context, base_name, globals_)
    return Emitted(kernel, emit_launcher(proto, launch))
  if plan.strategy == 'colprog':
    from .colprog import emit_colprog
    kernel, launch, extra = emit_colprog(chain, plan, context, base_name, globals_)
    return Emitted(kernel, emit_launcher(proto, launch), extra)
  if plan.strategy == 'dmma':
    from .dmma import emit_dmma
    kernel, launch, extra = emit_dmma(chain, plan, context, base_name, globals_)
    return Emitted(kernel, emit_launcher(proto, launch), extra)
  if plan.strategy == 'tcsplit':
    from .tcsplit import emit_tcsplit
    kernel, launch, extra = emit_tcsplit(chain, plan, context, base_name, globals_)
    return Emitted(kernel, emit_launcher(proto, launch), extra)
  raise ValueError(f'unknown strategy {plan.strategy}')
