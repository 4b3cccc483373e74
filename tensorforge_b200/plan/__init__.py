"""Tiling planner: choose how a lowered chain is mapped onto B200.

Strategies (one per code generator in tensorforge_b200.codegen):
  'generic'  every descriptor form the frontend accepts; each batch element is owned by
             a group of `threads_per_element` lanes, intermediates live in shared memory.
  'colprog'  column programs on CUDA cores for shared-left GEMM chains
             (out_e = sum_t A_t * B_e * R_{e,t}); one thread per output column.
  'tcsplit'  the same chains with the dense A_t * B_e stages on tcgen05 tensor cores as
             split (hi/lo) products accumulated in FP32 in tensor memory.
"""
from dataclasses import dataclass, field
from typing import Optional

from ..common.exceptions import GenerationError
from ..common.basic_types import FloatingPointType

SMEM_LIMIT = 227 * 1024


@dataclass
class Plan:
  strategy: str
  params: dict = field(default_factory=dict)
  smem_bytes: int = 0
  threads: int = 0
  note: str = ''

  def key(self):
    return f'{self.strategy}:' + ','.join(f'{k}={v}' for k, v in sorted(self.params.items()))


def generic_plan(chain, fp_size, threads_per_element=None, elements_per_block=None, points_per_lane=None):
  """Pick lanes per element and elements per CTA for the generic generator (and, for
  chains with elementwise stages, how many points a lane handles per pass)."""
  from ..codegen.generic import smem_layout
  ew_only = bool(chain.stages) and all(getattr(st, 'kind', '') == 'elementwise' for st in chain.stages)
  if ew_only and threads_per_element is None:
    # elementwise-only chains stream their operands: a warp per element and 8 elements per
    # CTA, 4 points per lane per pass, measured fastest on B200 (93 % of the copy bandwidth
    # for a 56x9 update, against 45 % with 256 lanes per element)
    threads_per_element = 32
    elements_per_block = 8 if elements_per_block is None else elements_per_block
  if threads_per_element is None:
    # measured on B200 over 1,973 random chains (sizes 4..128, 1-4 stages, lane groups of
    # 4..256): 256 lanes per element with one element per CTA is the fastest generic
    # variant for most chains (1,140 of them; the next, 256 x 2, for 237)
    threads_per_element = 256
  g = threads_per_element
  e = elements_per_block if elements_per_block is not None else 1
  while True:
    shared, per_elem = smem_layout(chain)
    total = (shared + per_elem * e) * fp_size
    if total <= SMEM_LIMIT or e == 1:
      break
    e = max(1, e // 2)
  if total > SMEM_LIMIT:
    raise GenerationError(f'chain needs {total} bytes of shared memory per element group')
  if g * e > 1024:
    e = max(1, 1024 // g)
  params = {'threads_per_element': g, 'elements_per_block': e}
  if chain.has_elementwise():
    params['points_per_lane'] = points_per_lane or 4
  return Plan('generic', params, total, g * e)


def make_plan(chain, context, variant=None):
  """Plan for `chain`; `variant` (a tuner's pick) overrides Options.variant."""
  opts = context.get_user_options()
  fp_size = context.fp_type.size()
  variant = variant or opts.variant or {}
  forced = variant.get('strategy')
  precision = opts.precision
  from . import chains as chainplan
  if forced in (None, 'colprog', 'tcsplit'):
    shape = chainplan.match_left_chain(chain)
    if shape is not None:
      if precision in ('tf32x3', 'bf16x3') and context.fp_type == FloatingPointType.FLOAT and forced != 'colprog':
        p = chainplan.tcsplit_plan(chain, shape, precision, variant)
        if p is not None:
          return p
        if forced == 'tcsplit':
          raise GenerationError('chain does not fit the tensor-core split form')
      # FP64: the DMMA tensor path is the default (exact FP64 products and sums, another
      # summation order); the column program stays available as a forced variant
      if precision in ('plain', 'dmma') and context.fp_type == FloatingPointType.DOUBLE and forced != 'colprog':
        p = chainplan.dmma_plan(chain, shape, variant)
        if p is not None:
          return p
      if forced != 'tcsplit':
        p = chainplan.colprog_plan(chain, shape, fp_size, variant)
        if p is not None:
          return p
    elif forced in ('colprog', 'tcsplit'):
      raise GenerationError(f'chain does not have the shared-left GEMM form required by {forced}')
  return generic_plan(chain, fp_size, variant.get('threads_per_element'), variant.get('elements_per_block'),
                      variant.get('points_per_lane'))
