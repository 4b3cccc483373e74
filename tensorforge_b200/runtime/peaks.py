"""Measured CUDA-core FMA peaks (FP32 / FP64) and the FP64 DMMA peak, timed with CUDA events."""
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
