"""Package surface used by yateto (tensorforge/interop.py:1-23)."""
import os

_HERE = os.path.dirname(os.path.realpath(__file__))


def get_cmake_path():
  return os.path.join(_HERE, 'share', 'cmake')


def print_cmake_path():
  print(get_cmake_path(), end='')


def get_routine_generator(yateto):
  from .frontend import yateto as fe
  return fe.YatetoFrontend


def get_version():
  with open(os.path.join(_HERE, 'VERSION')) as f:
    return f.read()


def print_version():
  print(get_version(), end='')


def use_fusedgemm_cost():
  return True
