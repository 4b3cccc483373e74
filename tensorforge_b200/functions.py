"""Elementwise expression builders under the reference's module name
(tensorforge/functions.py:1): `from tensorforge_b200.functions import *`."""
from .generators.optree import *  # noqa: F401,F403
