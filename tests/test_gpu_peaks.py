"""GPU: the roofline probes of the native runtime library return plausible rates."""
import pytest

pytestmark = pytest.mark.gpu


def test_fma_and_dmma_probes():
  from tensorforge_b200.runtime.peaks import fma_peak, dmma_peak
  assert 1e13 < fma_peak('float') < 2e14       # FP32 FFMA, B200: ~69 TFLOP/s measured
  assert 1e12 < dmma_peak() < 1e14             # FP64 DMMA, ~37 TFLOP/s measured


@pytest.mark.parametrize('n,a_smem', [(64, False), (128, False), (256, False), (64, True), (256, True)])
def test_tcgen05_tf32_probe(n, a_smem):
  from tensorforge_b200.runtime.peaks import tc_tf32_peak
  rate = tc_tf32_peak(n, a_smem, iters=4096)
  print(f'tcgen05 TF32 128x{n}x8, A from {"shared" if a_smem else "tensor"} memory: {rate / 1e12:.0f} TFLOP/s')
  assert 1e13 < rate < 3e15
