"""Autotuning: variant spaces, exhaustive measurement and the learned cost model.

  chains.py      seeded random contraction chains (the cost-model workload)
  variants.py    tunable variants of a chain and their 32-dim feature vectors
  autotune.py    builds every variant of a chain into one library, measures them on the GPU,
                 caches results per chain signature and GPU (resumable)
  cost_model.py  32-64-64-1 MLP on log-runtime, trained and evaluated on the GPU by the
                 hand-written kernels of csrc/mlp.cu; top-k selection and regret
"""
