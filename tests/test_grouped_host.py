"""Host logic of the per-group mixed-shape launch (no GPU): stream assignment."""
from tensorforge_b200.grouped import PerGroupLaunch


class _Chain:
  def __init__(self, flops):
    self.flops = flops

  def nz_flops_per_element(self):
    return self.flops


class _Gen:
  def __init__(self, flops):
    self.chain = _Chain(flops)

  def get_chain(self):
    return self.chain


class _Kernel:
  def __init__(self, flops):
    self.generator = _Gen(flops)


def test_largest_work_first_onto_least_loaded_stream():
  # work = elements x flops: 900, 500, 400, 300, 100, 0
  kernels = [_Kernel(f) for f in (1, 5, 4, 3, 1, 7)]
  kwargs = [{'numElements': n} for n in (900, 100, 100, 100, 100, 0)]
  pg = PerGroupLaunch(kernels, kwargs, streams=3)
  assert sorted(g for lane in pg.lanes for g in lane) == list(range(6))
  assert pg.lanes[0][0] == 0                    # the largest group leads its own stream
  work = [900, 500, 400, 300, 100, 0]
  # 900 -> s0, 500 -> s1, 400 -> s2, 300 -> s2 (400), 100 -> s1 (500), 0 -> s1 (600)
  assert [sum(work[g] for g in lane) for lane in pg.lanes] == [900, 600, 700]


def test_more_streams_than_groups():
  pg = PerGroupLaunch([_Kernel(1), _Kernel(2)], [{'numElements': 10}, {'numElements': 10}], streams=4)
  assert sorted(len(lane) for lane in pg.lanes) == [0, 0, 1, 1]
