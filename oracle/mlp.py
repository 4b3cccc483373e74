"""FP64 numpy restatement of the cost-model MLP (forward, loss, gradients).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). Same parameter layout as
tensorforge_b200/csrc/mlp.cu: W1[64][32], b1[64], W2[64][64], b2[64], W3[64], b3[1];
L = 1/(2B) sum_b (y_b - t_b)^2 with y = W3 relu(W2 relu(W1 x + b1) + b2) + b3.
"""
import numpy as np

IN, H = 32, 64
NPARAMS = H * IN + H + H * H + H + H + 1


def unpack(p):
  p = np.asarray(p, dtype=np.float64)
  o = 0
  W1 = p[o:o + H * IN].reshape(H, IN); o += H * IN
  b1 = p[o:o + H]; o += H
  W2 = p[o:o + H * H].reshape(H, H); o += H * H
  b2 = p[o:o + H]; o += H
  W3 = p[o:o + H]; o += H
  b3 = p[o]
  return W1, b1, W2, b2, W3, b3


def forward(p, X):
  W1, b1, W2, b2, W3, b3 = unpack(p)
  X = np.asarray(X, dtype=np.float64)
  h1 = np.maximum(X @ W1.T + b1, 0.0)
  h2 = np.maximum(h1 @ W2.T + b2, 0.0)
  return h2 @ W3 + b3, h1, h2


def loss(p, X, T):
  y, _, _ = forward(p, X)
  return 0.5 * np.mean((y - np.asarray(T, dtype=np.float64)) ** 2)


def grads(p, X, T):
  W1, b1, W2, b2, W3, b3 = unpack(p)
  X = np.asarray(X, dtype=np.float64)
  y, h1, h2 = forward(p, X)
  B = X.shape[0]
  dy = (y - np.asarray(T, dtype=np.float64)) / B
  dW3 = dy @ h2
  db3 = dy.sum()
  d2 = np.outer(dy, W3) * (h2 > 0)
  dW2 = d2.T @ h1
  db2 = d2.sum(0)
  d1 = (d2 @ W2) * (h1 > 0)
  dW1 = d1.T @ X
  db1 = d1.sum(0)
  return np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3, [db3]])


def init(seed=0):
  rng = np.random.default_rng(seed)
  W1 = rng.normal(0, np.sqrt(2.0 / IN), (H, IN))
  W2 = rng.normal(0, np.sqrt(2.0 / H), (H, H))
  W3 = rng.normal(0, np.sqrt(1.0 / H), H)
  return np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), W3, [0.0]]).astype(np.float32)
