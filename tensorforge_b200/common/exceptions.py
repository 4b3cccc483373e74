"""Generator error types (same names and meaning as tensorforge/common/exceptions.py:1-6)."""


class GenerationError(Exception):
  """The operation list cannot be lowered (bad shapes, unsupported form)."""


class InternalError(Exception):
  """A generator invariant was violated."""
