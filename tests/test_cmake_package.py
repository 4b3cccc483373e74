"""find_package(TensorForge) from a CMake project builds a generated kernel (no GPU)."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.skipif(shutil.which('cmake') is None or shutil.which('nvcc') is None,
                                reason='cmake and nvcc are needed')

CMAKE = '''cmake_minimum_required(VERSION 3.24)
project(tfb_cmake_probe LANGUAGES CXX CUDA)
find_package(TensorForge {version} REQUIRED)
add_library(generated STATIC generated.cu)
target_link_libraries(generated PRIVATE TensorForge::TensorForge)
set_target_properties(generated PROPERTIES CUDA_ARCHITECTURES ${{TensorForge_CUDA_ARCHITECTURES}})
'''


def _configure(tmp_path, version='', backend=None):
  from tensorforge_b200 import interop
  from tensorforge_b200.kernels import make
  g = make('c0_gemm_ptr', 'float')
  (tmp_path / 'generated.cu').write_text(g.get_source())
  (tmp_path / 'CMakeLists.txt').write_text(CMAKE.format(version=version))
  cmd = ['cmake', '-S', str(tmp_path), '-B', str(tmp_path / 'build'),
         f'-DCMAKE_PREFIX_PATH={interop.get_cmake_path()}', f'-DCMAKE_CUDA_COMPILER={shutil.which("nvcc")}']
  if backend:
    cmd.append(f'-DDEVICE_BACKEND={backend}')
  return subprocess.run(cmd, capture_output=True, text=True), g


def test_find_package_builds_a_generated_kernel(tmp_path):
  from tensorforge_b200 import interop
  conf, g = _configure(tmp_path, version=interop.get_version().strip())
  assert conf.returncode == 0, conf.stdout[-2000:] + conf.stderr[-2000:]
  build = subprocess.run(['cmake', '--build', str(tmp_path / 'build')], capture_output=True, text=True)
  assert build.returncode == 0, build.stdout[-3000:] + build.stderr[-2000:]
  assert os.path.exists(tmp_path / 'build' / 'libgenerated.a')
  # the archive holds the generated launcher and the runtime helpers
  nm = subprocess.run(['nm', str(tmp_path / 'build' / 'libgenerated.a')], capture_output=True, text=True).stdout
  assert f'launcher_{g.get_base_name()}' in nm
  assert 'tensorforge_last_status' in nm


def test_other_backends_are_rejected(tmp_path):
  conf, _ = _configure(tmp_path, backend='hip')
  assert conf.returncode != 0
  assert 'sm_100a only' in conf.stdout + conf.stderr
