"""Every C entry point declared under include/ is exported by the library that implements it.

Loads the libraries with ctypes and resolves the symbols only (no CUDA call, no GPU).
"""
import ctypes
import glob
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
  """Function names declared inside the header's extern "C" blocks (macros excluded)."""
  text = open(header).read()
  text = re.sub(r'//[^\n]*', '', text)
  text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
  text = '\n'.join(m.group(1) for m in re.finditer(r'extern "C" \{(.*?)\n\}', text, flags=re.S))
  lines, names = [], []
  cont = False
  for line in text.splitlines():  # drop #define bodies, including continued lines
    if cont or line.lstrip().startswith('#'):
      cont = line.rstrip().endswith('\\')
      continue
    lines.append(line)
  body = '\n'.join(lines)
  for m in re.finditer(r'^\s*(?:int|void|unsigned|size_t)\s*\*?\s*(\w+)\s*\(', body, flags=re.M):
    names.append(m.group(1))
  return names


def test_runtime_library_exports_its_headers():
  from tensorforge_b200.runtime import native
  native.build()
  lib = ctypes.CDLL(native.LIB, mode=ctypes.RTLD_LOCAL)
  checked = 0
  for header in ('tensorforge_b200_runtime.h', 'tensorforge_aux.h'):
    names = _declared(os.path.join(REPO, 'include', header))
    assert names, header
    for name in names:
      assert hasattr(lib, name), f'{name} ({header}) not exported by {native.LIB}'
      checked += 1
  assert checked == 11  # 9 runtime entry points + 2 status helpers


def test_headers_are_all_covered():
  # headers whose entry points are checked here (the grouped header declares per-set names)
  covered = {'tensorforge_b200_runtime.h', 'tensorforge_aux.h', 'tensorforge_b200_grouped.h'}
  assert {os.path.basename(h) for h in glob.glob(os.path.join(REPO, 'include', '*.h'))} == covered


def test_grouped_library_exports_declared_set_entry_points():
  from tensorforge_b200.kernels import grouped_catalogue
  gk = dict(grouped_catalogue())['test']
  lib = ctypes.CDLL(gk.build(), mode=ctypes.RTLD_LOCAL)
  text = open(os.path.join(REPO, 'include', 'tensorforge_b200_grouped.h')).read()
  for stem in re.findall(r'TFB_EXTERN_C int (\w+)##set\(', text):
    assert hasattr(lib, f'{stem}{gk.name}'), stem


def test_generated_launcher_exports_reference_name():
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime.build import build_library
  g = make('c0_gemm_ptr', 'float')
  lib = ctypes.CDLL(build_library(g.get_source()), mode=ctypes.RTLD_LOCAL)
  assert not hasattr(lib, f'launcher_{g.get_base_name()}')  # C++ linkage: the name is mangled
  assert hasattr(lib, f'tfb_launch_{g.get_base_name()}')  # the status-returning C form
  assert hasattr(lib, 'tensorforge_last_status')


def test_reference_declaration_links_against_generated_library(tmp_path):
  """A C++ caller written against the reference's header (tensorforge/generators/
  generator.py:198-199: `void launcher_<name>(...);`, C++ linkage, no extern "C")
  links against the generated library unchanged. Link only, no GPU call."""
  import shutil
  import subprocess
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime.build import build_library
  g = make('c0_gemm_ptr', 'float')
  so = build_library(g.get_source())
  args = ['nullptr' if '*' in t else '0' for t, _ in g.abi_params()]
  (tmp_path / 'caller.cpp').write_text(
    '#include <cstddef>\n' + g.get_header() +
    'int main(int argc, char**) {\n'
    f'  if (argc > 99) launcher_{g.get_base_name()}({", ".join(args)});\n'
    '  return 0;\n}\n')
  cxx = shutil.which('g++')
  if cxx is None:
    pytest.skip('g++ not found')
  r = subprocess.run([cxx, str(tmp_path / 'caller.cpp'), so, '-o', str(tmp_path / 'caller'),
                      '-Wl,--unresolved-symbols=ignore-in-shared-libs'], capture_output=True, text=True)
  assert r.returncode == 0, r.stderr[-3000:]
