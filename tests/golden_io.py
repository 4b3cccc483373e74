"""Load golden vectors and stage them on the GPU in the launcher's ABI layout."""
import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def golden_files():
  return sorted(glob.glob(os.path.join(GOLDEN, '*.npz')))


def load(path):
  z = np.load(path)
  meta = json.loads(bytes(z['meta']).decode())
  return z, meta


def golden_ids():
  return [os.path.basename(p)[:-4] for p in golden_files()]


def oracle_memory(z, meta):
  from oracle.multilinear import Memory
  mem = Memory()
  for s in meta['symbols']:
    n = s['name']
    if s['kind'] == 'scalar':
      mem.scalars[n] = float(z[f'scalar_{n}'])
      continue
    mem.buffers[n] = z[f'in_{n}'].astype(np.float64)
    if f'starts_{n}' in z:
      mem.starts[n] = z[f'starts_{n}']
  return mem


def device_args(z, meta, torch):
  """Device buffers + launcher keyword arguments for a golden case."""
  dt = torch.float32 if meta['fp'] == 'float' else torch.float64
  bufs, kwargs, keep = {}, {}, []
  for s in meta['symbols']:
    n = s['name']
    if s['kind'] == 'scalar':
      kwargs[n] = float(z[f'scalar_{n}'])
      continue
    b = torch.from_numpy(np.ascontiguousarray(z[f'in_{n}'])).to(dtype=dt, device='cuda')
    bufs[n] = b
    if s['kind'] == 'ptr':
      starts = z[f'starts_{n}'] - s['extra_offset']
      ptrs = torch.tensor(b.data_ptr() + starts.astype(np.int64) * b.element_size(), dtype=torch.int64, device='cuda')
      keep.append(ptrs)
      kwargs[n] = ptrs
      kwargs[f'{n}_extraOffset'] = s['extra_offset']
    elif s['kind'] == 'strided':
      kwargs[n] = b
      kwargs[f'{n}_extraOffset'] = s['extra_offset']
    else:
      kwargs[n] = b
  kwargs['numElements'] = int(z['n'])
  return bufs, kwargs, keep
