"""Measured CUDA-core FMA peaks (FP32 / FP64), the FP64 DMMA peak and the tcgen05 TF32 MMA rate,
timed with CUDA events."""
import ctypes


def fma_peak(dtype='float', iters=4096, reps=5):
  """Best-of-`reps` FLOP/s of the FMA probe in libtfb200_runtime.so."""
  import torch
  from . import native
  lib = native.load()
  fn = lib.tfb_fma_peak_launch
  fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
  fn.restype = ctypes.c_int
  sms = torch.cuda.get_device_properties(0).multi_processor_count
  blocks = sms * 8
  out = torch.zeros(blocks, dtype=torch.float64, device='cuda')
  stream = torch.cuda.current_stream()
  is_d = 1 if dtype == 'double' else 0
  fn(is_d, out.data_ptr(), 64, blocks, stream.cuda_stream)
  best = 0.0
  for _ in range(reps):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    rc = fn(is_d, out.data_ptr(), iters, blocks, stream.cuda_stream)
    e.record(stream)
    e.synchronize()
    if rc != 0:
      raise RuntimeError(f'FMA probe failed: CUDA error {rc}')
    secs = s.elapsed_time(e) / 1e3
    best = max(best, 2.0 * 16 * iters * blocks * 256 / secs)
  return best


def dmma_peak(iters=2048, reps=5):
  """Best-of-`reps` FLOP/s of the m8n8k4 FP64 tensor-core probe."""
  import torch
  from . import native
  lib = native.load()
  fn = lib.tfb_dmma_peak_launch
  fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
  fn.restype = ctypes.c_int
  sms = torch.cuda.get_device_properties(0).multi_processor_count
  blocks = sms * 8
  out = torch.zeros(blocks, dtype=torch.float64, device='cuda')
  stream = torch.cuda.current_stream()
  fn(out.data_ptr(), 32, blocks, stream.cuda_stream)
  best = 0.0
  for _ in range(reps):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    rc = fn(out.data_ptr(), iters, blocks, stream.cuda_stream)
    e.record(stream)
    e.synchronize()
    if rc != 0:
      raise RuntimeError(f'DMMA probe failed: CUDA error {rc}')
    secs = s.elapsed_time(e) / 1e3
    best = max(best, 512.0 * 8 * iters * blocks * 8 / secs)
  return best


def tc_tf32_peak(n=64, a_smem=False, iters=16384, reps=3):
  """Best-of-`reps` FLOP/s of back-to-back 128 x n x 8 tcgen05 TF32 MMAs, one CTA per SM
  (A from tensor memory, or from shared memory with a_smem)."""
  import torch
  from . import native
  lib = native.load()
  fn = lib.tfb_tc_tf32_peak_launch
  fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
  fn.restype = ctypes.c_int
  sms = torch.cuda.get_device_properties(0).multi_processor_count
  err = torch.zeros(1, dtype=torch.int32, device='cuda')
  stream = torch.cuda.current_stream()
  iters = iters // 8 * 8 + 1   # the probe issues 1 + 8 k MMAs
  rc = fn(n, int(a_smem), err.data_ptr(), 65, sms, stream.cuda_stream)
  if rc != 0:
    raise RuntimeError(f'tcgen05 TF32 probe failed: CUDA error {rc}')
  best = 0.0
  for _ in range(reps):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    rc = fn(n, int(a_smem), err.data_ptr(), iters, sms, stream.cuda_stream)
    e.record(stream)
    e.synchronize()
    if rc != 0:
      raise RuntimeError(f'tcgen05 TF32 probe failed: CUDA error {rc}')
    secs = s.elapsed_time(e) / 1e3
    best = max(best, 2.0 * 128 * n * 8 * iters * sms / secs)
  if int(err.item()) != 0:
    raise RuntimeError('tcgen05 TF32 probe: a bounded wait ran out')
  return best
