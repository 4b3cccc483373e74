"""Learned cost model: a 32-64-64-1 MLP predicting log-runtime of (chain, variant) pairs.

Training and inference run on the GPU through the hand-written kernels of
csrc/mlp.cu (tfb_mlp_forward / tfb_mlp_backward / tfb_mlp_loss / tfb_mlp_adam), exposed by
the native runtime library; parameters and optimiser state are FP32 device buffers.
Features are standardised with the training set's mean / std. `top_k` ranks a chain's
variants by predicted time; `regret` compares the measured best of the top k against the
exhaustive best.
"""
import ctypes
import json
import math

import numpy as np

NFEAT, HID = 32, 64


class CostModel:
  def __init__(self, seed=0):
    import torch
    from ..runtime import native
    self.lib = native.load()
    self._bind()
    self.nparams = self.lib.tfb_mlp_num_params()
    p = self._init_params(seed)
    self.params = torch.tensor(p, dtype=torch.float32, device='cuda')
    self.m = torch.zeros_like(self.params)
    self.v = torch.zeros_like(self.params)
    self.grads = torch.zeros_like(self.params)
    self.mean = np.zeros(NFEAT, np.float32)
    self.std = np.ones(NFEAT, np.float32)
    self.step = 0

  def _bind(self):
    L = self.lib
    vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.tfb_mlp_num_params.restype = i
    L.tfb_mlp_forward.argtypes = [vp, vp, i, vp, vp, vp, vp]
    L.tfb_mlp_backward.argtypes = [vp, vp, vp, i, vp, vp, vp, vp, vp, vp, vp, vp]
    L.tfb_mlp_loss.argtypes = [vp, vp, i, vp, vp]
    L.tfb_mlp_adam.argtypes = [vp, vp, vp, vp, i, f, f, f, f, i, vp]
    for fn in (L.tfb_mlp_forward, L.tfb_mlp_backward, L.tfb_mlp_loss, L.tfb_mlp_adam):
      fn.restype = i

  def _init_params(self, seed):
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0, math.sqrt(2.0 / NFEAT), (HID, NFEAT))
    W2 = rng.normal(0, math.sqrt(2.0 / HID), (HID, HID))
    W3 = rng.normal(0, math.sqrt(1.0 / HID), HID)
    return np.concatenate([W1.ravel(), np.zeros(HID), W2.ravel(), np.zeros(HID), W3, [0.0]]).astype(np.float32)

  @staticmethod
  def _check(rc, what):
    if rc != 0:
      raise RuntimeError(f'{what} failed with CUDA error {rc}')

  def _stream(self):
    import torch
    return torch.cuda.current_stream().cuda_stream

  # ---------------------------------------------------------------- raw kernel calls
  def forward(self, X, keep=False):
    """Predictions for device matrix X [B, 32] (already standardised)."""
    import torch
    B = X.shape[0]
    Y = torch.empty(B, dtype=torch.float32, device='cuda')
    H1 = torch.empty((B, HID), dtype=torch.float32, device='cuda') if keep else None
    H2 = torch.empty((B, HID), dtype=torch.float32, device='cuda') if keep else None
    self._check(self.lib.tfb_mlp_forward(self.params.data_ptr(), X.data_ptr(), B,
                                         H1.data_ptr() if keep else None, H2.data_ptr() if keep else None,
                                         Y.data_ptr(), self._stream()), 'mlp forward')
    return (Y, H1, H2) if keep else Y

  def gradients(self, X, T):
    """Loss and parameter gradients (device) for device batch X [B,32], targets T [B]."""
    import torch
    B = X.shape[0]
    Y, H1, H2 = self.forward(X, keep=True)
    dH1 = torch.empty_like(H1)
    dH2 = torch.empty_like(H2)
    dY = torch.empty_like(Y)
    self._check(self.lib.tfb_mlp_backward(self.params.data_ptr(), X.data_ptr(), T.data_ptr(), B, H1.data_ptr(),
                                          H2.data_ptr(), Y.data_ptr(), dH1.data_ptr(), dH2.data_ptr(),
                                          dY.data_ptr(), self.grads.data_ptr(), self._stream()), 'mlp backward')
    loss = torch.empty(1, dtype=torch.float32, device='cuda')
    self._check(self.lib.tfb_mlp_loss(Y.data_ptr(), T.data_ptr(), B, loss.data_ptr(), self._stream()), 'mlp loss')
    return loss, self.grads

  def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    self.step += 1
    self._check(self.lib.tfb_mlp_adam(self.params.data_ptr(), self.grads.data_ptr(), self.m.data_ptr(),
                                      self.v.data_ptr(), self.nparams, lr, b1, b2, eps, self.step,
                                      self._stream()), 'mlp adam')

  # ---------------------------------------------------------------- training / inference
  def fit(self, feats, log_ms, steps=3000, lr=2e-3, batch=4096, seed=0):
    """Train on host arrays feats [N,32], log_ms [N] (mini-batches sampled on the host)."""
    import torch
    feats = np.asarray(feats, np.float32)
    self.mean = feats.mean(0)
    self.std = feats.std(0) + 1e-6
    Xa = torch.tensor((feats - self.mean) / self.std, device='cuda')
    Ta = torch.tensor(np.asarray(log_ms, np.float32), device='cuda')
    rng = np.random.default_rng(seed)
    history = []
    n = Xa.shape[0]
    for it in range(steps):
      if n > batch:
        idx = torch.tensor(rng.choice(n, batch, replace=False), device='cuda')
        X, T = Xa[idx].contiguous(), Ta[idx].contiguous()
      else:
        X, T = Xa, Ta
      step_lr = lr * (0.1 ** (it / max(1, steps)))
      loss, _ = self.gradients(X, T)
      self.adam_step(step_lr)
      if it % 100 == 0 or it == steps - 1:
        history.append((it, float(loss.item())))
    return history

  def predict(self, feats):
    import torch
    X = torch.tensor((np.asarray(feats, np.float32) - self.mean) / self.std, device='cuda').contiguous()
    return self.forward(X).cpu().numpy()

  def save(self, path):
    np.savez(path, params=self.params.cpu().numpy(), mean=self.mean, std=self.std)

  def load(self, path):
    import torch
    z = np.load(path)
    self.params = torch.tensor(z['params'], device='cuda')
    self.mean, self.std = z['mean'], z['std']


def host_predict(params, mean, std, feats):
  """Predicted log-runtime on the host (numpy), for picking a variant at generation time,
  where no GPU need be present. Same parameter layout and arithmetic as tfb_mlp_forward."""
  p = np.asarray(params, np.float64)
  o = 0
  W1 = p[o:o + HID * NFEAT].reshape(HID, NFEAT); o += HID * NFEAT
  b1 = p[o:o + HID]; o += HID
  W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
  b2 = p[o:o + HID]; o += HID
  W3 = p[o:o + HID]; o += HID
  b3 = p[o]
  X = (np.asarray(feats, np.float64) - mean) / std
  h1 = np.maximum(X @ W1.T + b1, 0.0)
  h2 = np.maximum(h1 @ W2.T + b2, 0.0)
  return h2 @ W3 + b3


def top_k(pred_log_ms, k=5):
  return list(np.argsort(pred_log_ms)[:k])


def regret(measured_ms, picks):
  best = min(measured_ms)
  got = min(measured_ms[i] for i in picks)
  return (got - best) / best
