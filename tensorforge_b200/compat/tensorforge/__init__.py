"""`import tensorforge` for code written against the reference package (yateto, SeisSol's
code generators, user scripts): put this directory (tensorforge_b200/compat) on the Python
path and the reference's module paths resolve to tensorforge_b200's modules, e.g.

    from tensorforge.common.matrix.tensor import Tensor, SubTensor
    from tensorforge.generators.descriptions import GemmDescr
    from tensorforge.generators.generator import Generator

Each public module of the reference's frontend, descriptor, generator and interop layers
is registered under its reference name (sys.modules aliases), so the classes are the same
objects whichever name imports them. The reference's backend internals (backend/*, the
lexics, the hardware database) have no counterpart: the sm_100a generators replace them.
"""
import importlib
import sys
import types

_MODULES = [
  'common', 'common.aux', 'common.basic_types', 'common.context', 'common.exceptions', 'common.operation',
  'common.matrix', 'common.matrix.boundingbox', 'common.matrix.spp', 'common.matrix.tensor',
  'generators', 'generators.descriptions', 'generators.generator', 'generators.optree',
  'frontend', 'frontend.yateto', 'functions', 'interface', 'interop',
]

for _name in _MODULES:
  sys.modules[f'{__name__}.{_name}'] = importlib.import_module(f'tensorforge_b200.{_name}')
# the reference keeps the architecture description in common/vm/vm.py; here it is part of
# common/context.py (VM, vm_factory)
_vm_pkg = types.ModuleType(f'{__name__}.common.vm')
_vm_pkg.__path__ = []
_vm_pkg.vm = sys.modules['tensorforge_b200.common.context']
sys.modules[f'{__name__}.common.vm'] = _vm_pkg
sys.modules[f'{__name__}.common.vm.vm'] = _vm_pkg.vm
for _name in ('common', 'generators', 'frontend'):
  setattr(sys.modules[__name__], _name, sys.modules[f'{__name__}.{_name}'])

from tensorforge_b200.interop import *  # noqa: E402,F401,F403
