"""FP64 restatement of what a TensorForge-generated kernel computes, per batch element.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Follows the reference:
  * operand naming / ABI order: tensorforge/generators/generator.py:301-347
  * index ranges = intersection of operand bounding boxes:
    tensorforge/backend/instructions/compute/multilinear.py:58-96
  * per-element base address: tensorforge/backend/instructions/ptr_manip.py:39-65
  * dense entry address  sum_j (idx_j - bbox.lower_j) * stride_j  with column-major
    strides over the full shape: tensorforge/backend/symbol.py:304-312; a dense operand
    that has no output-leading index and no permutation is read through a contiguous
    copy of its bounding box, i.e. with strides over the box sizes:
    tensorforge/backend/instructions/builders/multilinear_builder.py:94-113 and
    tensorforge/backend/instructions/memory/load.py:76-137
  * sparse entry: compact value at spp.linear_index(idx - bbox.lower), zero when
    absent: tensorforge/backend/symbol.py:340-401, tensorforge/common/matrix/spp.py:84-109
  * `add` accumulates the previous destination value: multilinear.py:226-247
  * the store covers the computed index ranges only: memory/store.py:131-191
  * elements e < numElements with flags[e] != 0 (or no flags): generator.py:145-152, :501-505
"""
import numpy as np

NONE, STRIDED, PTR_BASED, SCALAR = 'none', 'strided', 'pointer_based', 'scalar'


def _addr_name(t):
  return str(t.addressing)


def _colmajor(sizes):
  out, acc = [], 1
  for s in sizes:
    out.append(acc)
    acc *= s
  return out


def name_operands(descr_list):
  """Return (all tensors in first-appearance order, ABI symbol list).

  Every non-temporary tensor is an ABI symbol (generator.py:330-347, :384-405); one
  carrying fewer than 16 compile-time values keeps its parameter, but the kernel uses
  the inlined values instead (generator.py:337-339).
  """
  seen = {}
  for d in descr_list:
    for sub in (d.matrix_list() if hasattr(d, 'oplist') else [d.dest] + list(d.ops)):
      seen.setdefault(id(sub.tensor), sub.tensor)
  tensors = list(seen.values())
  symbols = []
  for t in tensors:
    if t.is_tmp:
      continue
    symbols.append(t)
  return tensors, symbols


def _sparse_table(t):
  """{relative index tuple: storage position} of a compactly stored operand."""
  spp = t.spp
  mask = getattr(spp, 'indexmask', None)
  table = {}
  if mask is not None:
    for idx in zip(*np.nonzero(mask)):
      table[tuple(int(i) for i in idx)] = int(mask[idx]) - 1
    return table
  raise ValueError('unsupported sparsity pattern for compact storage')


def _is_sparse_storage(t):
  name = type(t.spp).__name__
  dense = t.spp.count_nz() == int(np.prod(t.shape)) if len(t.shape) else True
  return (not dense) and name != 'BoundingBoxSPP'


def _scalar_data_value(t, quirks):
  """Value of a rank-0 compile-time tensor.

  The reference looks values up by index tuple in `data` (tensor.py:57-62); a plain list
  such as GemmDescr's `[alpha]` has no `()` key, so the reference reads 0. With
  quirks=False the intended value (the list's single entry) is used.
  """
  d = t.data
  if isinstance(d, dict):
    return float(d.get((), 0.0))
  if quirks:
    return 0.0
  return float(d[0])


class Memory:
  """Flat buffers for the ABI symbols plus per-element start offsets.

  buffers[name]  : 1-D float64 array (a copy of the device buffer)
  starts[name]   : int array of length N (start of element e, extra offset included)
                   or None for shared operands
  scalars[name]  : float for SCALAR symbols
  """

  def __init__(self):
    self.buffers = {}
    self.starts = {}
    self.scalars = {}


def _stored_targets(d):
  """Per operand, the index of each *stored* dimension: target[i][v] names view dimension v,
  which is stored dimension permute[i][v] (descriptions.py:126-149 expresses GEMM
  transposes this way; the reference generator stops with NameError on such permutes)."""
  out = []
  for i, tgt in enumerate(d.target):
    perm = d.permute[i] if d.permute is not None and i < len(d.permute) else None
    if not perm or len(perm) != len(tgt) or sorted(perm) != list(range(len(tgt))):
      out.append(list(tgt))
      continue
    eff = [0] * len(tgt)
    for v, sdim in enumerate(perm):
      eff[sdim] = tgt[v]
    out.append(eff)
  return out


def evaluate(descr_list, memory: Memory, num_elements: int, flags=None, quirks=True, fp32=False):
  """Run the chain on every allowed element, updating memory.buffers in place.

  Elementwise descriptors run through oracle/elementwise.py (`fp32` applies to them).
  """
  tensors, symbols = name_operands(descr_list)
  sym_names = {}
  for i, t in enumerate(symbols):
    sym_names[id(t)] = f'm{i}'
  tmp_counter = 0
  tmp_names = {}
  for t in tensors:
    if t.is_tmp:
      tmp_names[id(t)] = f't{tmp_counter}'
      tmp_counter += 1

  elems = np.arange(num_elements)
  if flags is not None:
    elems = elems[np.asarray(flags)[:num_elements] != 0]
  ne = len(elems)
  tmp_values = {}   # id(tensor) -> (ranges, array [ne, *sizes])

  for d in descr_list:
    if hasattr(d, 'oplist'):
      from .elementwise import evaluate_elementwise
      evaluate_elementwise(d, memory, elems, sym_names, tmp_values, fp32=fp32)
      continue
    targets = _stored_targets(d)
    # index ranges
    nr, kr = {}, {}
    for sub, tgt in zip(d.ops, targets):
      for j, t in enumerate(tgt):
        lo, up = sub.bbox.lower()[j], sub.bbox.upper()[j]
        table, key = (nr, t) if t >= 0 else (kr, -t - 1)
        if key in table:
          table[key] = (max(table[key][0], lo), min(table[key][1], up))
        else:
          table[key] = (lo, up)
    n_ranges = [nr[t] for t in range(len(nr))]
    k_ranges = [kr[k] for k in range(len(kr))]
    letters_n = 'abcdefgh'
    letters_k = 'pqrstuvw'

    operands, subs = [], []
    for i_op, (sub, tgt) in enumerate(zip(d.ops, targets)):
      t = sub.tensor
      box = [n_ranges[x] if x >= 0 else k_ranges[-x - 1] for x in tgt]
      sizes = [u - l for l, u in box]
      grids = np.meshgrid(*[np.arange(l, u) for l, u in box], indexing='ij') if box else []
      spec = ''.join(letters_n[x] if x >= 0 else letters_k[-x - 1] for x in tgt)
      if t.is_tmp:
        rng, arr = tmp_values[id(t)]
        sl = tuple(slice(l - r0, u - r0) for (l, u), (r0, _) in zip(box, rng))
        vals = arr[(slice(None),) + sl]
      elif t.data is not None and len(t.data) < 16 and len(tgt) == 0:
        vals = np.full((ne,), _scalar_data_value(t, quirks))
      elif _addr_name(t) == SCALAR:
        vals = np.full((ne,), float(memory.scalars[sym_names[id(t)]]))
      elif t.data is not None and len(t.data) < 16:
        # compile-time data tensor (fewer than 16 values)
        vals = np.zeros([ne] + sizes)
        for pos in np.ndindex(*sizes):
          idx = tuple(l + p for (l, _), p in zip(box, pos))
          v = t.value(idx) if isinstance(t.data, dict) else None
          vals[(slice(None),) + pos] = 0.0 if v is None else v
      else:
        name = sym_names[id(t)]
        buf = memory.buffers[name]
        base = np.zeros(ne, dtype=np.int64) if _addr_name(t) == NONE else np.asarray(memory.starts[name])[elems]
        lower = t.bbox.lower()
        if _is_sparse_storage(t):
          table = _sparse_table(t)
          pos_arr = np.full(sizes, -1, dtype=np.int64)
          for p in np.ndindex(*sizes):
            rel = tuple(l + q - lo for (l, _), q, lo in zip(box, p, lower))
            pos_arr[p] = table.get(rel, -1)
          gathered = buf[(base.reshape([-1] + [1] * len(sizes)) + np.maximum(pos_arr, 0)[None])]
          vals = np.where(pos_arr[None] >= 0, gathered, 0.0)
        else:
          perm = d.permute[i_op] if d.permute is not None else list(range(len(tgt)))
          compact = list(perm) == list(range(len(tgt))) and (0 not in tgt)
          strides = _colmajor(t.bbox.sizes() if compact else list(t.shape))
          off = np.zeros(sizes, dtype=np.int64)
          for g, lo, st in zip(grids, lower, strides):
            off = off + (g - lo) * st
          vals = buf[base.reshape([-1] + [1] * len(sizes)) + off[None]]
      operands.append(vals)
      subs.append('z' + spec)
    out_spec = 'z' + ''.join(letters_n[t] for t in range(len(n_ranges)))
    result = np.einsum(','.join(subs) + '->' + out_spec, *operands, optimize=True) if operands else None

    dest = d.dest.tensor
    if dest.is_tmp:
      if d.add and id(dest) in tmp_values:
        rng, prev = tmp_values[id(dest)]
        result = result + prev
      tmp_values[id(dest)] = (n_ranges, result)
    else:
      name = sym_names[id(dest)]
      buf = memory.buffers[name]
      base = np.asarray(memory.starts[name])[elems]
      sizes = [u - l for l, u in n_ranges]
      grids = np.meshgrid(*[np.arange(l, u) for l, u in n_ranges], indexing='ij')
      off = np.zeros(sizes, dtype=np.int64)
      for g, lo, st in zip(grids, dest.bbox.lower(), _colmajor(list(dest.shape))):
        off = off + (g - lo) * st
      addr = base.reshape([-1] + [1] * len(sizes)) + off[None]
      if d.add:
        result = result + buf[addr]
      buf[addr] = result
  return memory
