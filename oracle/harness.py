"""Seeded operand buffers laid out exactly as the launcher ABI expects.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

For a descriptor list and element count N this builds one flat buffer per ABI symbol:
  NONE       the shared operand (its stored values)
  STRIDED    N slots of volume(shape) values, element e at e*volume + extraOffset
             (tensorforge/backend/instructions/ptr_manip.py:37-45)
  PTR_BASED  N slots in a shuffled order, pointer e -> slot perm[e]; the element's data
             starts extraOffset values after the pointer (ptr_manip.py:46-51)
  SCALAR     a value passed by value
"""
import numpy as np
from .multilinear import name_operands, Memory, _is_sparse_storage


class SymbolLayout:
  def __init__(self, name, tensor, kind, size, starts, extra_offset, slot):
    self.name = name
    self.tensor = tensor
    self.kind = kind            # 'shared' | 'strided' | 'ptr' | 'scalar'
    self.size = size            # buffer length in values
    self.starts = starts        # np.int64[N] or None
    self.extra_offset = extra_offset
    self.slot = slot            # values per PTR_BASED slot


def storage_values(t):
  """Values one copy of `t` occupies: compact nonzeros if sparse, else the full volume."""
  if _is_sparse_storage(t):
    mask = t.spp.indexmask
    return int(mask.max())
  return int(np.prod(t.shape)) if len(t.shape) else 1


def make_layout(descrs, n, seed=0, extra_offsets=True):
  rng = np.random.default_rng(seed + 7777)
  _, symbols = name_operands(descrs)
  layouts = []
  for i, t in enumerate(symbols):
    name = f'm{i}'
    addr = str(t.addressing)
    if addr == 'scalar':
      layouts.append(SymbolLayout(name, t, 'scalar', 0, None, 0, 0))
      continue
    store = storage_values(t)
    if addr == 'none':
      layouts.append(SymbolLayout(name, t, 'shared', store, None, 0, 0))
      continue
    off = int(rng.integers(0, 5)) if extra_offsets else 0
    vol = int(np.prod(t.shape)) if len(t.shape) else 1
    if addr == 'strided':
      starts = np.arange(n, dtype=np.int64) * vol + off
      size = n * vol + off + 4
      layouts.append(SymbolLayout(name, t, 'strided', size, starts, off, vol))
    else:
      slot = store + off + 3
      perm = rng.permutation(n)
      starts = perm.astype(np.int64) * slot + off
      size = n * slot
      layouts.append(SymbolLayout(name, t, 'ptr', size, starts, off, slot))
  return layouts


def make_values(size, rng, dist='uniform'):
  if dist == 'uniform':
    return rng.uniform(-1.0, 1.0, size)
  if dist == 'loguniform':
    mag = 10.0 ** rng.uniform(-3.0, 3.0, size)
    return mag * np.where(rng.random(size) < 0.5, -1.0, 1.0)
  if dist == 'int':
    return rng.integers(-4, 5, size).astype(np.float64)
  raise ValueError(dist)


def make_memory(descrs, n, seed=0, dist='uniform', extra_offsets=True, dtype=np.float32):
  """Return (layouts, Memory) with float64 buffers holding values exactly representable in `dtype`."""
  layouts = make_layout(descrs, n, seed, extra_offsets)
  rng = np.random.default_rng(seed)
  mem = Memory()
  for lay in layouts:
    if lay.kind == 'scalar':
      mem.scalars[lay.name] = float(np.asarray(rng.uniform(0.5, 1.5), dtype=dtype))
      continue
    vals = make_values(lay.size, rng, dist).astype(dtype).astype(np.float64)
    mem.buffers[lay.name] = vals
    mem.starts[lay.name] = lay.starts
  return layouts, mem


def make_flags(n, seed=0, keep=0.75):
  rng = np.random.default_rng(seed + 31)
  return (rng.random(n) < keep).astype(np.uint32)
