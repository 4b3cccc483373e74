"""Seeded random contraction chains for tuning and for training the cost model.

A chain has 1..4 GEMM stages over one batch element. It starts from a per-element dense
operand X_0 (K_1 x N_0); stage s either multiplies from the left by a shared sparse matrix
(T_s = A_s * T_{s-1}, A_s is M_s x rows(T_{s-1})) or from the right by a per-element sparse
matrix (T_s = T_{s-1} * R_s, R_s is cols(T_{s-1}) x N_s), so each stage's contracted size is
the previous stage's M or N. Sizes are uniform over 4..128, operand densities uniform over
0.1..1.0, the batch log-uniform over 1e4..1e6 (capped so that no per-element operand array
exceeds `max_bytes`). The last stage writes the per-element output.
"""
from dataclasses import dataclass, field
from typing import List

import numpy as np


@dataclass
class StageSpec:
  side: str          # 'left' (shared A) or 'right' (per-element R)
  rows: int          # M of the stage result
  cols: int          # N of the stage result
  k: int             # contracted size
  density: float


@dataclass
class ChainSpec:
  index: int
  x_rows: int
  x_cols: int
  x_density: float
  stages: List[StageSpec]
  batch: int
  seed: int

  def key(self):
    parts = [f'{self.x_rows}x{self.x_cols}'] + [f'{s.side[0]}{s.rows}x{s.cols}k{s.k}d{s.density:.2f}' for s in self.stages]
    return f'c{self.index}:' + '-'.join(parts) + f'@{self.batch}'


def random_chains(n, seed=0, lo=4, hi=128, max_bytes=256 << 20):
  rng = np.random.default_rng(seed)
  out = []
  for i in range(n):
    L = int(rng.integers(1, 5))
    rows, cols = int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1))
    x = (rows, cols)
    stages = []
    for _ in range(L):
      d = float(rng.uniform(0.1, 1.0))
      if rng.random() < 0.5:
        m = int(rng.integers(lo, hi + 1))
        stages.append(StageSpec('left', m, cols, rows, d))
        rows = m
      else:
        nn = int(rng.integers(lo, hi + 1))
        stages.append(StageSpec('right', rows, nn, cols, d))
        cols = nn
    batch = int(round(np.exp(rng.uniform(np.log(1e4), np.log(1e6)))))
    # cap the batch so that the largest per-element operand array stays within max_bytes
    biggest = max([x[0] * x[1]] + [s.rows * s.cols for s in stages] +
                  [s.k * s.cols for s in stages if s.side == 'right']) * 4
    batch = max(64, min(batch, max_bytes // biggest))
    out.append(ChainSpec(i, x[0], x[1], 1.0, stages, batch, int(rng.integers(0, 2**31 - 1))))
  return out


def build_descriptors(spec: ChainSpec, ns):
  """Descriptor list (frontend API of namespace `ns`) computing the chain per element."""
  rng = np.random.default_rng(spec.seed)

  def pattern(r, c, d):
    mask = rng.random((r, c)) < d
    if not mask.any():
      mask[0, 0] = True
    return [(int(i), int(j)) for j in range(c) for i in range(r) if mask[i, j]]

  A = ns.Addressing
  cur = ns.Tensor([spec.x_rows, spec.x_cols], A.STRIDED)
  descrs = []
  for si, st in enumerate(spec.stages):
    last = si == len(spec.stages) - 1
    dest = ns.Tensor([st.rows, st.cols], A.STRIDED) if last else None
    if st.side == 'left':
      spp = ns.ListSPP(pattern(st.rows, st.k, st.density), (st.rows, st.k)) if st.density < 0.999 else None
      other = ns.Tensor([st.rows, st.k], A.NONE, spp=spp)
      ops = [ns.SubTensor(other), ns.SubTensor(cur)]
    else:
      spp = ns.ListSPP(pattern(st.k, st.cols, st.density), (st.k, st.cols)) if st.density < 0.999 else None
      other = ns.Tensor([st.k, st.cols], A.STRIDED, spp=spp)
      ops = [ns.SubTensor(cur), ns.SubTensor(other)]
    target = [[0, -1], [-1, 1]]
    if dest is None:
      dest = ns.generate_tmp_tensor(ops, target)
    descrs.append(ns.MultilinearDescr(ns.SubTensor(dest), ops, target, [[0, 1], [0, 1]]))
    cur = dest
  return descrs
