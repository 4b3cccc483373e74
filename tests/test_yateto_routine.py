"""The yateto routine file plus the gateway's call site compile for sm_100a as one
translation unit (no GPU); tests/test_gpu_yateto_routine.py runs it."""


def test_routine_and_call_site_compile(tmp_path):
  from tensorforge_b200.runtime.build import build_library
  from tests.yateto_routine import generate_routine
  g, _, source = generate_routine(tmp_path)
  assert 'yateto_execute' in source and f'launcher_{g.get_base_name()}(' in source
  build_library(source)
