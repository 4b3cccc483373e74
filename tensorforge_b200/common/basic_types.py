"""Enumerations shared by the frontend and the code generator.

Mirrors tensorforge/common/basic_types.py:4-169: the enum names, values and string
spellings are part of the interface (yateto passes them through), so they are kept.
"""
import enum


class DataFlowDirection(enum.Enum):
  SOURCE = 0
  SINK = 1
  SOURCESINK = 2


class Addressing(enum.Enum):
  """How one operand is found for batch element `e` (tensorforge/common/basic_types.py:9-48).

  NONE      one array shared by every element
  STRIDED   element e starts at e * volume(shape) (+ extra offset)
  PTR_BASED element e starts at ptrs[e] (+ extra offset); ptrs is a device array of pointers
  SCALAR    a value passed to the launcher by value
  """
  NONE = 0
  STRIDED = 1
  PTR_BASED = 2
  SCALAR = 3

  @classmethod
  def addr2ptr_type(cls, addr_type):
    return {Addressing.NONE: '*', Addressing.STRIDED: '*',
            Addressing.PTR_BASED: '**', Addressing.SCALAR: ''}[addr_type]

  @classmethod
  def str2addr(cls, string):
    table = {'none': Addressing.NONE, 'strided': Addressing.STRIDED,
             'pointer_based': Addressing.PTR_BASED, 'scalar': Addressing.SCALAR}
    if string not in table:
      raise ValueError(f'arg must be either none, strided, pointer_based, or scalar; given: {string}')
    return table[string]

  @classmethod
  def addr2str(cls, addr):
    return {Addressing.NONE: 'none', Addressing.STRIDED: 'strided',
            Addressing.PTR_BASED: 'pointer_based', Addressing.SCALAR: 'scalar'}[addr]

  def __str__(self):
    return self.addr2str(self)

  def to_pointer(self):
    return self.addr2ptr_type(self)


class StridedAddressing:
  """Strided addressing with an explicit offset and stride (basic_types.py:50-59)."""

  def __init__(self, offset, stride=None):
    self.offset = offset
    self.stride = stride

  def to_pointer(self):
    return Addressing.STRIDED.to_pointer()


class FloatingPointType(enum.Enum):
  FLOAT = 0
  DOUBLE = 1
  HALF = 2
  BFLOAT16 = 3
  BOOL = 10
  INT = 20
  UINT = 21
  LONG = 22
  ULONG = 23

  def size(self):
    return {FloatingPointType.FLOAT: 4, FloatingPointType.DOUBLE: 8, FloatingPointType.HALF: 2,
            FloatingPointType.BFLOAT16: 2, FloatingPointType.BOOL: 1, FloatingPointType.INT: 4,
            FloatingPointType.UINT: 4, FloatingPointType.LONG: 8,
            FloatingPointType.ULONG: 8}[self]

  def __str__(self):
    return self.as_str(self)

  def literal(self, value):
    if self == FloatingPointType.FLOAT:
      return f'{float(value):.9e}f'
    if self == FloatingPointType.DOUBLE:
      return f'{float(value):.17e}'
    if self == FloatingPointType.HALF:
      return f'static_cast<__half>({float(value):.9e})'
    if self == FloatingPointType.BFLOAT16:
      return f'static_cast<__nv_bfloat16>({float(value):.9e})'
    if self == FloatingPointType.BOOL:
      return 'true' if value else 'false'
    if self == FloatingPointType.INT:
      return f'{int(value)}'
    if self == FloatingPointType.UINT:
      return f'{int(value)}u'
    if self == FloatingPointType.LONG:
      return f'{int(value)}L'
    return f'{int(value)}UL'

  @classmethod
  def as_str(cls, fp):
    return {FloatingPointType.FLOAT: 'float', FloatingPointType.DOUBLE: 'double',
            FloatingPointType.HALF: 'half', FloatingPointType.BFLOAT16: 'bfloat16',
            FloatingPointType.BOOL: 'bool', FloatingPointType.INT: 'int',
            FloatingPointType.LONG: 'long', FloatingPointType.UINT: 'unsigned int',
            FloatingPointType.ULONG: 'unsigned long'}[fp]

  @classmethod
  def str2enum(cls, as_str: str):
    return {'float': FloatingPointType.FLOAT, 'double': FloatingPointType.DOUBLE,
            'half': FloatingPointType.HALF, 'bfloat16': FloatingPointType.BFLOAT16,
            'bool': FloatingPointType.BOOL, 'int': FloatingPointType.INT,
            'long': FloatingPointType.LONG, 'unsigned int': FloatingPointType.UINT,
            'unsigned long': FloatingPointType.ULONG}[as_str]

  @classmethod
  def ytt2enum(cls, as_str: str):
    return {'f32': FloatingPointType.FLOAT, 'f64': FloatingPointType.DOUBLE,
            'f16': FloatingPointType.HALF, 'bf16': FloatingPointType.BFLOAT16,
            'bool': FloatingPointType.BOOL, 'i8': FloatingPointType.INT,
            'i16': FloatingPointType.INT, 'i32': FloatingPointType.INT,
            'i64': FloatingPointType.LONG, 'u32': FloatingPointType.UINT,
            'u64': FloatingPointType.ULONG}[as_str]


class GeneralLexicon:
  """Fixed identifiers of the emitted code and launcher ABI (basic_types.py:157-169)."""
  BATCH_ID_NAME = 'batchId'
  NUM_ELEMENTS = 'numElements'
  EXTRA_OFFSET = '_extraOffset'
  STREAM_PTR_STR = 'streamPtr'
  ALPHA_SYMBOL_NAME = 'alpha'
  BETA_SYMBOL_NAME = 'beta'
  FLAGS_NAME = 'flags'
  GLOBAL_MEM_PREFIX = 'glb_'
  TOTAL_SHR_MEM = 'totalShrMem'
  LOCAL_SHR_MEM = 'localShrMem'
  SHR_MEM_REGION_PREFIX = 'shrRegion'
  REG_NAME = 'reg'
