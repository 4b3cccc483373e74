"""Host-resident batches through a generated kernel with transfers overlapped by compute.

A launcher call works on device buffers. For batches that live in (pinned) host memory,
`HostPipeline` cuts the batch into slices of whole elements and sends each slice through
one of a few CUDA streams, round robin: host->device copies of the slice's batched inputs,
the launcher on the slice (its pointer arguments advanced to the slice's first element,
numElements = the slice's length), device->host copy of the slice's output. The copy of
slice c+1 in, the kernel on slice c and the copy of slice c-1 out then run at the same
time (two copy engines and the SMs). Shared operands are copied once per call, before the
first slice. Elements are independent, so the result equals one launch over the batch.

The side streams wait for the caller's current stream at the start of a call, and the
caller's stream waits for all of them at the end, so consecutive calls and work queued by
the caller stay ordered; timing with events on the caller's stream covers the whole call.
Batched operands must be STRIDED (pointer-array operands would need per-slice pointer
arrays); flags are not supported. A compactly stored sparse input fills only the start of
each element's slot; only that part is copied (one 2D copy per slice through the native
runtime's `tfb_copy_rows_async`), which for the order-6 chain's S operands (24 of 81 values)
cuts the host->device bytes per element from 2,988 to 2,304.
"""


class HostPipeline:
  def __init__(self, kernel, generator, slices=8, streams=3):
    import torch
    self.kernel = kernel
    self.slices = max(1, int(slices))
    self.streams = [torch.cuda.Stream() for _ in range(max(1, int(streams)))]
    self.batched, self.shared, self.outputs = [], [], []
    # values the kernel reads per element, for compactly stored (sparse) batched operands
    self.used = {o.name: o.storage_size() for o in generator.get_chain().operands
                 if o.kind == 'batched' and o.sparse and o.storage_size() < o.element_volume()}
    for t, _ in generator.abi_symbols():
      a = t.addressing.name
      if a == 'PTR_BASED':
        raise ValueError(f'{t.name}: pointer-array operands are not supported by HostPipeline')
      if a == 'STRIDED':
        self.batched.append((t.name, t.get_real_volume()))
        if t.direction.name != 'SOURCE':
          self.outputs.append(t.name)
      elif a == 'NONE':
        self.shared.append(t.name)
    self.inputs = [n for n, _ in self.batched if n not in self.outputs or self._reads(generator, n)]

  @staticmethod
  def _reads(generator, name):
    """Outputs that the chain also reads (accumulated into) must be copied in as well."""
    for t, _ in generator.abi_symbols():
      if t.name == name:
        return t.direction.name != 'SINK'
    return False

  def __call__(self, host, device, num_elements, **scalars):
    """host / device: ABI name -> pinned host tensor / device tensor of the same layout
    (extra offsets are 0). Copies inputs in, runs the kernel, copies outputs out."""
    import torch
    cur = torch.cuda.current_stream()
    start = torch.cuda.Event()
    start.record(cur)
    for s in self.streams:
      s.wait_event(start)
    first = self.streams[0]
    with torch.cuda.stream(first):
      for name in self.shared:
        device[name].copy_(host[name], non_blocking=True)
    shared_done = torch.cuda.Event()
    shared_done.record(first)
    for s in self.streams[1:]:
      s.wait_event(shared_done)
    n = int(num_elements)
    step = -(-n // self.slices)
    vol = dict(self.batched)
    for c, e0 in enumerate(range(0, n, step)):
      e1 = min(n, e0 + step)
      s = self.streams[c % len(self.streams)]
      with torch.cuda.stream(s):
        for name in self.inputs:
          v = vol[name]
          if name in self.used:
            self._copy_rows(device[name], host[name], e0, e1, v, self.used[name], s)
          else:
            device[name][e0 * v:e1 * v].copy_(host[name][e0 * v:e1 * v], non_blocking=True)
        args = dict(scalars)
        for name, v in self.batched:
          d = device[name]
          args[name] = d.data_ptr() + e0 * v * d.element_size()
        for name in self.shared:
          args[name] = device[name]
        self.kernel(numElements=e1 - e0, streamPtr=s.cuda_stream, **args)
        for name in self.outputs:
          v = vol[name]
          host[name][e0 * v:e1 * v].copy_(device[name][e0 * v:e1 * v], non_blocking=True)
    for s in self.streams:
      done = torch.cuda.Event()
      done.record(s)
      cur.wait_event(done)

  @staticmethod
  def _copy_rows(dev, host, e0, e1, vol, used, stream):
    """Host -> device: the first `used` values of each of the slots e0..e1-1 (`vol` apart)."""
    import ctypes
    from . import native
    es = dev.element_size()
    lib = native.load()
    fn = lib.tfb_copy_rows_async
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                   ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p]
    err = fn(dev.data_ptr() + e0 * vol * es, vol * es, host.data_ptr() + e0 * vol * es, vol * es,
             used * es, e1 - e0, 1, stream.cuda_stream)
    if err != 0:
      raise RuntimeError(f'tfb_copy_rows_async failed with CUDA error {err}')
