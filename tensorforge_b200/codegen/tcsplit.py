"""tcgen05 split-precision generator for shared-left GEMM chains (sm_100a tensor cores).

Computes out_e = sum_t A_t * B_{e,t} * R_{e,t} (the chains of plan.chains) as

    out^T[(e,j), i] = sum_t sum_l U_t[l, (e,j)] * A_t[i, l],   U_t = B_{e,t} * R_{e,t}

one MMA chain per tile of TE = floor(128 / N) whole elements (TE*N flat output columns):
  * M = 128 rows = flat columns (e, j) (one TMEM lane each), N = rows of out padded to 16,
    K = sum_t K_t (each term padded to the MMA K step);
  * A operand (U^T, per element) lives in tensor memory. Per tile, the batched operands
    are fetched one tile ahead into a shared-memory stage (see the pipelines below); one
    producer thread per (element, row l)
    computes row l of U_t = B_e * R_{e,t} for all j with R_t's compile-time pattern
    unrolled and writes it to a padded transposition buffer; then each lane reads its
    column (e, j), splits it into hi + lo and writes both with tcgen05.st;
  * B operand (A_t^T, shared) is split once per CTA into hi + lo and kept in shared memory
    in the canonical no-swizzle K-major layout (8x16-byte core matrices);
  * the epilogue reads the accumulators with tcgen05.ld, stages the tile's output in
    shared memory and writes it with one bulk copy (cp.async.bulk, shared -> global) when
    the output is strided, 16-byte aligned and unmasked; otherwise each lane stores its
    own column.

Precisions: 'tf32x3' (kind::tf32: hi = value rounded to nearest TF32, lo = the rounded
remainder, so value = hi + lo to ~2^-24 and both are exact TF32 inputs), 'bf16x3'
(kind::f16 with BF16 inputs: hi = bf16(value), lo = bf16(value - hi); ~16 significant
bits, relative error ~1e-5, reported, not used where 1e-6 is required).

Accumulation: hi*hi products accumulate in one TMEM accumulator and the cross terms
hi*lo + lo*hi in a second one; the epilogue adds them in FP32. Every tensor-core
accumulation step rounds relative to its accumulator, so keeping the small cross terms
apart cuts the rounding error on the output by the share of MMAs they account for (2/3).

Pipelining: A has one TMEM slot per term; mbarriers hand slots between the producer warps
(4 groups of 4 warps sharing the 4 TMEM lane quadrants) and the MMA-issuing thread, so
the tensor cores work on tile n while the producers compute tile n+1; tile n's epilogue
then frees the accumulators for tile n+1. Every mbarrier wait is bounded: on timeout the
kernel records an error code (read with tfb_kernel_error_<name>) and exits after
releasing its tensor memory.

Producer pipelines (plan option `pipe`):
  2 (default when it fits in shared memory): one input stage, filled by one bulk copy
    (cp.async.bulk global -> this CTA's shared memory) per contiguous, 16-byte aligned B block
    and cp.async for the R blocks, completion tracked by a stage mbarrier (expect_tx bytes
    plus one cp.async arrival per producer); one U pass computes U_t for every term (B's
    row loaded once) into one transposition buffer per term; the previous tile's output
    is staged over the consumed B block and written with one bulk store. Three named
    barriers per tile.
  1: the original per-term pipeline (double-buffered cp.async stage, U phase and lane
    phase per term, two transposition buffers); used when pipe 2 does not fit.
The bulk B copy is issued by producer 0 after its output bulk store has read the stage;
when a B block is not contiguous or not 16-byte aligned, every producer copies it with
cp.async after one more barrier.
"""
from .. import plan as _plan
from ..plan import Plan
from ..plan.chains import match_left_chain

KSTEP = {'tf32x3': 8, 'bf16x3': 16}
ESIZE = {'tf32x3': 4, 'bf16x3': 2}
H_GROUPS = 4


def _pad(x, m):
  return (x + m - 1) // m * m


def layout(shape, precision):
  ks = KSTEP[precision]
  es = ESIZE[precision]
  n_mma = _pad(shape.M, 16)
  kpad = [_pad(t.K, ks) for t in shape.terms]
  a_cols = [kp * es // 4 for kp in kpad]          # TMEM columns per split per term
  slot_cols = [2 * c for c in a_cols]               # hi + lo
  tmem_used = sum(slot_cols) + 2 * n_mma            # + main and correction accumulators
  b_bytes = sum(2 * n_mma * kp * es for kp in kpad)  # hi + lo, all terms
  te = 128 // shape.N if shape.N <= 128 else 0
  return dict(ks=ks, es=es, n_mma=n_mma, kpad=kpad, a_cols=a_cols, slot_cols=slot_cols,
              tmem_used=tmem_used, b_bytes=b_bytes, te=te)


def staged_operands(shape):
  """Distinct batched operands a tile stages: [(operand, values per element)]."""
  seen = []
  for t in shape.terms:
    for op, vals in ((t.B, t.B.element_volume()), (t.R, t.R.storage_size() if t.R is not None else 0)):
      if op is None or op.kind != 'batched':
        continue
      if all(op is not o for o, _ in seen):
        seen.append((op, vals))
  return seen


def smem_plan(shape, precision):
  lay = layout(shape, precision)
  te = lay['te']
  tc = te * shape.N
  stage = sum(te * _pad(v, 4) * 4 for _, v in staged_operands(shape))
  kmax = max(t.K for t in shape.terms)
  pitch = _pad(kmax, 4) + 4
  ubuf = max(tc * pitch * 4, tc * shape.M * 4)
  b_bytes = lay['b_bytes']
  off_stage = _pad(b_bytes, 128)
  off_u = off_stage + 2 * _pad(stage, 128)
  # two transposition buffers (term t uses buffer t % 2) when they fit: saves a barrier per term
  nbuf = 2 if off_u + 2 * _pad(ubuf, 128) + 256 <= 227 * 1024 else 1
  off_bar = off_u + nbuf * _pad(ubuf, 128)
  total = off_bar + 256
  return dict(off_stage=off_stage, stage=_pad(stage, 128), off_u=off_u, pitch=pitch, nbuf=nbuf,
              ubuf_bytes=_pad(ubuf, 128), off_bar=off_bar, total=total, te=te, tc=tc)


def _bulk_eligible(op, vals):
  """A tile of this operand is one contiguous block: one bulk copy when aligned at run time."""
  return op.addressing.name == 'STRIDED' and op.element_volume() == vals and (vals * 4) % 16 == 0


def smem_plan_v2(shape, precision, l64=False):
  """Shared memory of the one-pass pipeline: single input stage (B blocks first, the tile's
  output staged over them, R blocks behind both) and one transposition buffer per term."""
  lay = layout(shape, precision)
  te = lay['te']
  tc = te * shape.N
  b_ops = []
  for t in shape.terms:
    if all(t.B is not o for o in b_ops):
      b_ops.append(t.B)
  r_ops = [op for op, _ in staged_operands(shape) if all(op is not o for o in b_ops)]
  stage_off = {}
  off = 0
  for op in b_ops:
    stage_off[op.name] = off
    off += te * _pad(op.element_volume(), 4)
  off = _pad(max(off, te * shape.out.element_volume()), 4)
  for op in r_ops:
    stage_off[op.name] = off
    off += te * _pad(op.storage_size() if op.sparse else op.element_volume(), 4)
  stage = _pad(off * 4, 128)
  kmax = max(t.K for t in shape.terms)
  # transposition rows: 16-byte aligned for the lane phase's 128-bit loads, or (l64) a pitch
  # of 2 mod 32 words so that 16 consecutive rows fall on distinct bank pairs for 64-bit loads
  pitch = _pad(kmax, 4) + 4
  if l64:
    # row r's 64-bit word w sits on bank pair (r * pitch / 2 + w) mod 16: pitch / 2 odd
    pitch = _pad(kmax, 2) + (2 if (_pad(kmax, 2) // 2) % 2 == 0 else 0)
  ubuf = _pad(tc * pitch * 4, 128)
  off_stage = _pad(lay['b_bytes'], 128)
  off_u = off_stage + stage
  off_bar = off_u + len(shape.terms) * ubuf
  total = off_bar + 256
  return dict(off_stage=off_stage, stage=stage, stage_off=stage_off, b_ops=b_ops, r_ops=r_ops, off_u=off_u,
              pitch=pitch, ubuf_bytes=ubuf, off_bar=off_bar, total=total, te=te, tc=tc)


def smem_plan_v3(shape, precision, qreg=False, fuse=False, rbuf2=False, opad=False, l64=False):
  """Shared memory of the warp-specialised pipeline: the one-pass layout, an output staging
  buffer for the epilogue warps' bulk stores (32 rows per warp, or 16 rows at a time when
  only that fits) and the B operand. Without `fuse` B is stored for the real output rows
  only (rows M..N_mma-1 of the MMA's B tile then read the next block and land in
  accumulator columns the epilogue never reads); with `fuse` each term's hi and lo blocks
  are whole N_mma-row tiles, back to back, read by one MMA of width 2 N_mma."""
  sm = smem_plan_v2(shape, precision, l64)
  if qreg:
    # the stage holds the R blocks only (B is read into registers)
    off = 0
    stage_off = {}
    for op in sm['r_ops']:
      stage_off[op.name] = off
      off += sm['te'] * _pad(op.storage_size() if op.sparse else op.element_volume(), 4)
    stage = _pad(off * 4, 128)
    shrink = sm['stage'] - stage
    sm = dict(sm, stage=stage, stage_off=stage_off, off_u=sm['off_u'] - shrink, off_bar=sm['off_bar'] - shrink,
              total=sm['total'] - shrink)
  lay = layout(shape, precision)
  rows_b = lay['n_mma'] if fuse else _pad(shape.M, 8)
  b_bytes = sum(2 * rows_b * kp * lay['es'] for kp in lay['kpad'])
  shift = sm['off_stage'] - _pad(b_bytes, 128)
  out = dict(sm, rows_b=rows_b, b_bytes=b_bytes, ost_rows=0)
  for k in ('off_stage', 'off_u', 'off_bar', 'total'):
    out[k] = sm[k] - shift
  if rbuf2:
    # a second buffer for the R blocks (the loader fetches them one tile ahead)
    rstart = min(sm['stage_off'][op.name] for op in sm['r_ops'])
    rend = max(sm['stage_off'][op.name] + sm['te'] * _pad(op.storage_size() if op.sparse else op.element_volume(), 4)
               for op in sm['r_ops'])
    rbytes = _pad((rend - rstart) * 4, 128)
    out['off_rbuf1'] = out['off_bar']
    out['rbuf_delta'] = (out['off_rbuf1'] - out['off_stage']) // 4 - rstart
    out['off_bar'] += rbytes
    out['total'] += rbytes
  if shape.M % 4 == 0:
    out['ost_pitch'] = shape.M + 4 if opad else shape.M
    for rows in (32, 16):
      ost = _pad(4 * rows * out['ost_pitch'] * 4, 128)
      if out['total'] + ost <= _plan.SMEM_LIMIT:
        out['off_ost'] = out['off_bar']
        out['off_bar'] += ost
        out['total'] += ost
        out['ost_rows'] = rows
        break
  return out


def direct_ok(shape):
  """The direct-lane producers need one per-element B operand shared by every term, an R
  factor (batched, sparse or dense) in every term, all with the same K and P."""
  t0 = shape.terms[0]
  if t0.B is None or t0.B.kind != 'batched':
    return False
  for t in shape.terms:
    if t.B is not t0.B or t.R is None or t.R.kind != 'batched' or t.K != t0.K or t.P != t0.P:
      return False
  return True


def smem_plan_direct(shape, precision):
  """Shared memory of the direct-lane producers: the B operand's hi / lo tiles (whole
  N_mma-row tiles, back to back, for the fused MMA), two stages of the tile's per-element B
  blocks, two dense pair buffers of the R factors (value (m, j) of term t for flat column
  c = e * N + j at pair (t * P + m) * 128 + c, both halves the value, zeros outside the
  pattern written once) and the output staging buffer."""
  lay = layout(shape, precision)
  te = lay['te']
  tc = te * shape.N
  t0 = shape.terms[0]
  B = t0.B
  bvals = _pad(B.element_volume(), 4)
  stage = _pad(te * bvals * 4, 128)
  r_ops = []
  for t in shape.terms:
    if all(t.R is not o for o in r_ops):
      r_ops.append(t.R)
  rows_b = lay['n_mma']
  b_bytes = sum(2 * rows_b * kp * lay['es'] for kp in lay['kpad'])
  off_stage = _pad(b_bytes, 128)
  sd_bytes = _pad(len(shape.terms) * t0.P * 128 * 8, 128)
  off_sd = off_stage + 2 * stage
  off = off_sd + 2 * sd_bytes
  out = dict(off_stage=off_stage, stage=stage, stage_off={B.name: 0}, b_ops=[B], r_ops=r_ops,
             sdelta=stage // 4, off_sd=off_sd, sd_bytes=sd_bytes, sd_delta=sd_bytes // 8, rows_b=rows_b,
             b_bytes=b_bytes, te=te, tc=tc, ost_rows=0, pitch=0, off_u=off, ubuf_bytes=0, bvals=bvals)
  if shape.M % 4 == 0:
    out['ost_pitch'] = shape.M
    for rows in (32, 16):
      ost = _pad(4 * rows * shape.M * 4, 128)
      if off + ost + 256 <= _plan.SMEM_LIMIT:
        out['off_ost'] = off
        off += ost
        out['ost_rows'] = rows
        break
  out['off_bar'] = off
  out['total'] = off + 256
  return out


def pipe3_ok(shape, precision, chunk=16):
  """The warp-specialised pipeline (pipe 3) needs TF32 splits, a U pass for every term
  (K a multiple of 4, lane phases of at most 4 x 16 columns) and tensor memory for two A
  slots plus two accumulator pairs."""
  if precision != 'tf32x3' or chunk != 16:
    return False
  lay = layout(shape, precision)
  if any(t.R is None or t.R.kind != 'batched' or t.K % 4 for t in shape.terms):
    return False
  if any(-(-kp // 16) > H_GROUPS for kp in lay['kpad']):
    return False
  return 4 * max(lay['a_cols']) + 4 * lay['n_mma'] <= 512 or (
    2 * len(shape.terms) * max(lay['a_cols']) + 2 * lay['n_mma'] <= 512)


def plan(chain, shape, precision, variant):
  if precision not in KSTEP:
    return None
  # operand form B (codegen/tcsplit_b.py): the default for single-term chains (a plain GEMM
  # per element: 3.75e8 against 2.59e8 el/s for form U on 1M 56x56 x 56x9 pointer-array
  # GEMMs), opt-in otherwise (variant {'form': 'b'}): on the order-6 chain it measured 3.0e8
  # (13-element tiles, one B buffer) and 3.7e8 el/s (8-element tiles, two B buffers) against
  # 4.8e8 for form U below
  if 'form' in variant:
    form = variant['form']
  elif 'pipe' in variant or 'chunk' in variant or 'ahead' in variant:
    form = 'u'
  else:
    form = 'b' if len(shape.terms) == 1 else 'u'
  if precision == 'tf32x3' and form == 'b':
    # operand form B (codegen/tcsplit_b.py) when every term reads the same per-element input
    from .tcsplit_b import layout_b
    acc, bbuf, ws = int(variant.get('acc', 1)), int(variant.get('bbuf', 1)), int(variant.get('ws', 0))
    if ws:
      bbuf = 2   # the split team runs ahead of the tensor cores
    lb = layout_b(shape, acc, bbuf, variant.get('te'), ws)
    if lb is not None:
      params = {'precision': precision, 'form': 'b', 'acc': acc, 'bbuf': bbuf, 'te': lb['te']}
      if ws:
        params['ws'] = 1
      return Plan('tcsplit', params, max(lb['total'], 120 * 1024), 32 * (4 * H_GROUPS + 1),
                  note=f'form B: M={shape.M} N={shape.N} terms={len(shape.terms)} tile={lb["te"]} smem={lb["total"]}')
    if variant.get('form') == 'b':
      return None
  if shape.M > 256 or shape.N > 128:
    return None
  lay = layout(shape, precision)
  if lay['tmem_used'] > 512 or lay['te'] < 1:
    return None
  for t in shape.terms:
    if t.R is not None and t.R.kind != 'batched':
      return None
  default_pipe = 3 if (pipe3_ok(shape, precision, variant.get('chunk', 16)) and not variant.get('ahead')) else 2
  pipe = variant.get('pipe', default_pipe)
  if pipe == 3 and not pipe3_ok(shape, precision, variant.get('chunk', 16)):
    pipe = 2
  fuse = 0
  if pipe == 3:
    # defaults of the warp-specialised pipeline (measured on the order-6 chain, 500,000
    # elements: 6.37e8 el/s against 6.28e8 without the fused MMA and the bulk loader warp,
    # 5.67e8 with one U row per producer): two U rows per producer, the hi*hi and hi*lo
    # products as one MMA of twice the width when the whole B tiles fit
    qreg = bool(int(variant.get('qreg', 0)))
    fuse = int(variant.get('fuse', 1 if smem_plan_v3(shape, precision, qreg, True)['total'] <= _plan.SMEM_LIMIT else 0))
  # loader warp default: 3 (B blocks and the next tile's R blocks) when the second R buffer
  # fits, else 2
  rbuf2_fits = (pipe == 3 and not int(variant.get('qreg', 0))
                and smem_plan_v3(shape, precision, False, bool(fuse), True)['total'] <= _plan.SMEM_LIMIT)
  loader_default = 3 if rbuf2_fits else 2
  rbuf2 = rbuf2_fits and int(variant.get('loader', loader_default)) == 3
  opad = pipe == 3 and bool(int(variant.get('opad', 0)))
  direct = pipe == 3 and bool(int(variant.get('direct', 0))) and direct_ok(shape) and not int(variant.get('qreg', 0))
  if direct:
    fuse, rbuf2, opad = 1, False, False
    sm = smem_plan_direct(shape, precision)
  else:
    l64 = pipe == 3 and bool(int(variant.get('l64', 0)))
    sm = ((lambda sh, pr: smem_plan_v3(sh, pr, bool(int(variant.get('qreg', 0))), bool(fuse), rbuf2, opad, l64))
          if pipe == 3 else smem_plan_v2)(shape, precision) if pipe in (2, 3) else None
  if sm is None or sm['total'] > _plan.SMEM_LIMIT:
    pipe = 1
    sm = smem_plan(shape, precision)
  smem = max(sm['total'], 120 * 1024)  # one CTA per SM: it owns the SM's tensor memory
  if smem > _plan.SMEM_LIMIT:
    return None
  chunk = variant.get('chunk', 16)
  params = {'precision': precision, 'chunk': chunk, 'pipe': pipe}
  if int(variant.get('ahead', 0)) and pipe == 2:
    params['ahead'] = 1
  if pipe == 3:
    # A slots: one per term when the tensor memory also holds one accumulator pair (no
    # lane phase then waits for a slot), else two slots and two accumulator pairs
    lay3 = layout(shape, precision)
    scols = 2 * max(lay3['a_cols'])
    dcols = 2 * lay3['n_mma']
    nt = len(shape.terms)
    fit_one = nt * scols + dcols <= 512
    ns = int(variant.get('slots', nt if fit_one else 2))
    if ns not in (2, nt) or ns * scols + (1 if ns == nt else 2) * dcols > 512:
      ns = 2
    params['slots'] = ns
    # loader warp: 3 (default) issues the bulk copy of the B blocks and fetches the R blocks
    # of the next tile into the other of two R buffers (order-6 chain, 500,000 elements:
    # 6.44e8 el/s against 6.36e8 with mode 2); 2 issues only the bulk copy of the B blocks,
    # the producers keep the small R copies; 1 fetches all inputs into the one stage
    # (measured slower: 4.8e8 el/s, one warp issues the R copies slowly); 0 none
    params['loader'] = int(variant.get('loader', loader_default))
    if params['loader'] == 3 and not rbuf2:
      params['loader'] = 2
    if direct:
      # direct-lane producers: each producer thread computes its own TMEM lane's columns of
      # U_t from the B block (packed FMAs over the dense R pairs) and stores them to tensor
      # memory; loader mode 4 double-buffers the B stage and scatters the R factors
      params['direct'] = 1
      params['loader'] = 4
    # option: the per-element B operand goes straight from global memory into registers one
    # tile ahead (two rows per producer), so the stage only holds the R blocks
    b_ops = {id(t.B) for t in shape.terms}
    if (int(variant.get('qreg', 0)) and not params['loader'] and len(b_ops) == 1
        and all(t.K % 2 == 0 for t in shape.terms)
        and lay3['te'] * shape.terms[0].K // 2 <= 128 * H_GROUPS):
      params['qreg'] = 1
      params['urows'] = 2
  if pipe == 3 and fuse:
    # hi*hi and hi*lo as one MMA of twice the width (B's hi and lo tiles back to back, the
    # main and correction accumulators side by side)
    params['fuse'] = 1
  if (int(variant.get('urows', 2 if pipe == 3 else 1)) == 2 and pipe in (2, 3) and not direct
      and all(t.K % 2 == 0 for t in shape.terms)):
    params['urows'] = 2
  if pipe == 3 and int(variant.get('sleep', 4)):
    # waiting threads sleep in try_wait (global-timer bound) instead of spinning, leaving
    # the issue slots to the producers (order-6 chain, 500,000 elements: 6.51e8 el/s with
    # every role sleeping against 6.45e8 spinning); 3 keeps the MMA thread spinning, so it
    # issues as soon as a lane phase arrives (6.61e8 against 6.58e8 with every role
    # sleeping and 6.46e8 with the producers spinning too, option 2); the default 4 also
    # lets the producers poll 32 times before they sleep, so a phase that completes soon
    # costs no wake-up (6.93e8 against 6.79e8 with option 3)
    params['sleep'] = int(variant.get('sleep', 4))
  if opad:
    # option: output staging rows padded by 16 bytes (no bank conflicts on the staging
    # stores), each row written by its own bulk copy (measured slower: 6.44e8 el/s against
    # 6.51e8 with one bulk copy per 16 rows)
    params['opad'] = 1
  if pipe == 3 and int(variant.get('l64', 0)) and not direct:
    # option: the lane phase reads the transposition rows with 64-bit loads (rows of a pitch
    # that keeps 16 consecutive rows on distinct bank pairs)
    params['l64'] = 1
  if pipe == 3 and int(variant.get('uwarp', 1)) and not direct:
    # U pass work items aligned to warps, so no warp straddles two elements (order-6 chain,
    # 500,000 elements: 6.59e8 el/s against 6.51e8 with items spread over all threads)
    params['uwarp'] = 1
  if pipe == 3 and int(variant.get('lpk', 1)):
    # the lane phase forms lo = u - hi with packed FMAs (exact) and stores 16 columns per
    # tensor-memory store (order-6 chain, 500,000 elements: 6.76e8 el/s against 6.63e8 with
    # scalar subtractions and 8-column stores)
    params['lpk'] = 1
  if pipe == 3 and int(variant.get('epk', 1)):
    # the epilogue sums the main and correction accumulators with packed adds (6.81e8 el/s
    # against 6.77e8 with scalar adds)
    params['epk'] = 1
  if pipe == 3 and int(variant.get('estg', 0)):
    # option: the epilogue reads the accumulators in 16x256b fragments and stores whole
    # 32-byte sectors straight to global memory (no output staging; measured slower: 6.51e8
    # against 6.59e8 el/s with the staging buffer and bulk copies)
    params['estg'] = 1
  if pipe == 3 and int(variant.get('oswz', 0)):
    # option: the output staging stores of rows 4r..4r+3 (r odd) swap each chunk pair
    # (measured no gain: 6.57e8 against 6.58e8 el/s)
    params['oswz'] = 1
  if pipe == 3 and not int(variant.get('ostage', 1)):
    # option: the epilogue warps store their columns straight from registers (no staging)
    params['ostage'] = 0
  if int(variant.get('wait_probe', 0)) > 0:
    # failure-detection check: the kernel first waits, with this many polls, on an mbarrier
    # that nothing arrives on, records error 30 and returns before issuing any copy or MMA
    params['wait_probe'] = int(variant['wait_probe'])
  if int(variant.get('wait_probe_ns', 0)) > 0:
    # the same check for the sleeping wait: it gives up after this many nanoseconds of the
    # global timer
    params['wait_probe_ns'] = int(variant['wait_probe_ns'])
  return Plan('tcsplit', params, smem, 32 * (4 * H_GROUPS + 1),
              note=f'M={shape.M} N={shape.N} terms={len(shape.terms)} tmem={lay["tmem_used"]} smem={sm["total"]}')


HELPERS = r'''
#ifndef TFB_TCGEN05_HELPERS
#define TFB_TCGEN05_HELPERS
#include <cuda_bf16.h>
namespace tfb_tc {
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" :: "r"(smem_u32(bar)) : "memory");
}
// bounded wait on phase `parity`; returns false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long limit) {
  unsigned addr = smem_u32(bar);
  for (unsigned long long it = 0; it < limit; ++it) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(addr), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}
// bounded wait on phase `parity` that lets the thread sleep inside try_wait (the suspend-time
// hint, in ns) until the phase completes, so a waiting warp issues few instructions; returns
// false once `limit_ns` nanoseconds of the global timer have passed since the first poll
__device__ __forceinline__ bool mbar_wait_s(uint64_t* bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned addr = smem_u32(bar);
  const unsigned hint_ns = 1000000u;
  unsigned long long t0 = 0;
  for (;;) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(addr), "r"(parity), "r"(hint_ns) : "memory");
    if (ok) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t0 == 0) t0 = t;
    else if (t - t0 > limit_ns) return false;
  }
}
// a few polls without a suspend hint first (a phase that completes within them costs no
// wake-up), then the sleeping wait
__device__ __forceinline__ bool mbar_wait_h(uint64_t* bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned addr = smem_u32(bar);
  for (int i = 0; i < 32; ++i) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(addr), "r"(parity) : "memory");
    if (ok) return true;
  }
  return mbar_wait_s(bar, parity, limit_ns);
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void named_sync(unsigned id, unsigned n) { asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(n) : "memory"); }
// barrier over `n` threads that also returns the OR of `v` over them (same answer for all)
__device__ __forceinline__ bool any_sync(unsigned id, unsigned n, bool v) {
  unsigned r;
  asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}"
               : "=r"(r) : "r"((unsigned)v), "r"(id), "r"(n) : "memory");
  return r != 0;
}
__device__ __forceinline__ void tmem_alloc(unsigned* dst_smem, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ uint64_t smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo & 0x3FFFFu) >> 4) << 16;
  d |= (uint64_t)((sbo & 0x3FFFFu) >> 4) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for tcgen05
  return d;                 // base offset 0, no swizzle (layout type 0)
}
__device__ __forceinline__ void mma_tf32(unsigned d_tmem, unsigned a_tmem, uint64_t b_desc, unsigned idesc, unsigned accum) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}"
               :: "r"(d_tmem), "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accum) : "memory");
}
__device__ __forceinline__ void mma_f16(unsigned d_tmem, unsigned a_tmem, uint64_t b_desc, unsigned idesc, unsigned accum) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}"
               :: "r"(d_tmem), "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accum) : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void st_x8(unsigned taddr, const unsigned* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
               :: "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]) : "memory");
}
__device__ __forceinline__ void st_x16(unsigned taddr, const unsigned* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
               :: "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
                  "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]) : "memory");
}
__device__ __forceinline__ void st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void ld_x8(unsigned taddr, unsigned* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr) : "memory");
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 16 lanes x 256 bits from [taddr]: thread t receives words 2 (t % 4), 2 (t % 4) + 1 of lanes
// t / 4 (v[0], v[1]) and t / 4 + 8 (v[2], v[3])
__device__ __forceinline__ void ld16x256(unsigned taddr, unsigned* v) {
  asm volatile("tcgen05.ld.sync.aligned.16x256b.x1.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "r"(taddr) : "memory");
}
// round to nearest TF32 (10 stored mantissa bits); the result is exactly representable
__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// x = hi + lo with both parts exactly representable in TF32 up to |x| * 2^-24
__device__ __forceinline__ void tf32_split(float x, unsigned& hi, unsigned& lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
               :: "l"(gdst), "r"(smem_u32(ssrc)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// global -> this CTA's shared memory bulk copy, completion counted in bytes on `bar`
__device__ __forceinline__ void bulk_load(void* sdst, const void* gsrc, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :: "r"(smem_u32(sdst)), "l"(gsrc), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}"
               :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// arrive on `bar` once this thread's earlier cp.async copies have landed (counts as an arrival)
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
}  // namespace tfb_tc
#endif
'''


def emit_tcsplit(chain, plan_, context, base_name, globals_):
  shape = match_left_chain(chain)
  if plan_.params.get('form') == 'b':
    from .tcsplit_b import _TCB
    return _TCB(chain, shape, plan_, context, base_name).emit(globals_)
  return _TC(chain, shape, plan_, context, base_name).emit(globals_)


class _TC:
  WAIT_LIMIT = 1 << 26         # polls of a spinning wait
  WAIT_NS = 2000000000         # nanoseconds of a sleeping wait

  def __init__(self, chain, shape, plan_, ctx, base):
    self.chain = chain
    self.s = shape
    self.plan = plan_
    self.ctx = ctx
    self.base = base
    self.prec = plan_.params['precision']
    self.lay = layout(shape, self.prec)
    self.pipe = plan_.params.get('pipe', 1)
    self.qreg = self.pipe == 3 and int(plan_.params.get('qreg', 0)) == 1
    self.fuse = self.pipe == 3 and int(plan_.params.get('fuse', 0)) == 1
    self.rbuf2 = self.pipe == 3 and int(plan_.params.get('loader', 0)) == 3 and not self.qreg
    self.opad = self.pipe == 3 and bool(int(plan_.params.get('opad', 0)))
    self.direct = self.pipe == 3 and bool(int(plan_.params.get('direct', 0)))
    self.l64 = self.pipe == 3 and bool(int(plan_.params.get('l64', 0))) and not self.direct
    self.oswz = self.pipe == 3 and bool(int(plan_.params.get('oswz', 0)))
    self.estg = self.pipe == 3 and bool(int(plan_.params.get('estg', 0)))
    self.sm = (smem_plan_direct(shape, self.prec) if self.direct else
               smem_plan_v3(shape, self.prec, self.qreg, self.fuse, self.rbuf2, self.opad, self.l64) if self.pipe == 3 else
               smem_plan_v2(shape, self.prec) if self.pipe == 2 else smem_plan(shape, self.prec))
    self.LC = plan_.params['chunk']
    self.ahead = bool(plan_.params.get('ahead', 0))
    self.H = H_GROUPS
    self.lines = []
    self.ind = 0

  def w(self, s=''):
    self.lines.append('  ' * self.ind + s)

  def open(self, head):
    self.w(head + ' {')
    self.ind += 1

  def close(self):
    self.ind -= 1
    self.w('}')

  def params(self, globals_):
    params = []
    for t, _ in globals_:
      dt = 'float' if t.datatype is None else str(t.datatype)
      if t.addressing.name == 'SCALAR':
        params.append(f'{dt} {t.name}')
      else:
        const = 'const ' if t.direction.name == 'SOURCE' else ''
        params.append(f'{const}{dt}{t.addressing.to_pointer()} __restrict__ {t.name}')
        if t.addressing.name != 'NONE':
          params.append(f'unsigned {t.name}_extraOffset')
    params += ['size_t numElements', 'const unsigned* __restrict__ flags']
    return params

  def _elem_ptr(self, op, e):
    a = op.addressing.name
    if a == 'STRIDED':
      return f'({op.name} + ({e}) * {op.element_volume()}u + {op.name}_extraOffset)'
    if a == 'PTR_BASED':
      return f'({op.name}[{e}] + {op.name}_extraOffset)'
    return f'{op.name}'

  # ------------------------------------------------------------------ emit
  def emit(self, globals_):
    s, lay, sm, b = self.s, self.lay, self.sm, self.base
    kname = f'kernel_{b}'
    prec = self.prec
    n_mma = lay['n_mma']
    es = lay['es']
    H = self.H
    NP = 128 * H                       # producer threads
    nterms = len(s.terms)
    te, tcols = sm['te'], sm['tc']
    staged = staged_operands(s)
    stage_off = {}
    off = 0
    for op, vals in staged:
      stage_off[op.name] = off          # floats, within one stage buffer
      off += te * _pad(vals, 4)
    if self.pipe in (2, 3):
      stage_off = dict(sm['stage_off'])
    # B operand blocks (hi/lo per term) at the start of shared memory
    ke = 16 // es
    b_off = []
    off = 0
    rows_b = sm.get('rows_b', n_mma)   # B rows stored (the MMA's N tile reads n_mma)
    self.rows_b = rows_b
    for kp in lay['kpad']:
      b_off.append((off, off + rows_b * kp * es))
      off += 2 * rows_b * kp * es
    gathers = []
    for ti, t in enumerate(s.terms):
      kp = lay['kpad'][ti]
      look = t.A.sparse_lookup() if t.A.sparse else None
      tbl = []
      for n in range(rows_b):
        for k in range(kp):
          if n < t.A.shape[0] and k < t.K:
            tbl.append(k * t.A.shape[0] + n if look is None else look.get((n, k), -1))
          else:
            tbl.append(-1)
      gathers.append(tbl)

    self.w(HELPERS)
    self.w(f'// generated by tensorforge_b200 (strategy: tcsplit, {prec}, chunk={self.LC}, '
           f'tile={te} elements, smem={sm["total"]} B)')
    self.w('// meta data:')
    for o in self.chain.operands:
      self.w(f'// {o.tensor.gen_descr()}')
    for st in self.chain.stages:
      self.w(f'// {st.descr}')
    for ti, tbl in enumerate(gathers):
      self.w(f'__device__ const short bgather{ti}_{b}[{len(tbl)}] = {{{", ".join(str(x) for x in tbl)}}};')
    if self.direct:
      self._sd_table_decl()
    self.w(f'__device__ unsigned tfb_err_{b} = 0u;')
    self.w(f'extern "C" int tfb_kernel_error_{b}(void* stream) {{')
    self.w('  unsigned v = 0, z = 0;')
    self.w('  cudaStream_t st = static_cast<cudaStream_t>(stream);')
    self.w(f'  cudaMemcpyFromSymbolAsync(&v, tfb_err_{b}, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);')
    self.w(f'  cudaMemcpyToSymbolAsync(tfb_err_{b}, &z, sizeof(unsigned), 0, cudaMemcpyHostToDevice, st);')
    self.w('  cudaStreamSynchronize(st);')
    self.w('  return (int)v;')
    self.w('}')
    fmt = 2 if prec == 'tf32x3' else 1
    idesc = (1 << 4) | (fmt << 7) | (fmt << 10) | ((n_mma >> 3) << 17) | ((128 >> 4) << 24)
    smem = max(self.plan.smem_bytes, sm['total'])
    self.plan.smem_bytes = smem
    slot_base = []
    col = 0
    for ti in range(nterms):
      slot_base.append(col)
      col += lay['slot_cols'][ti]
    d_main, d_corr = col, col + n_mma
    p3 = self.pipe == 3
    # waits that sleep in try_wait (bounded by the global timer) or spin (bounded by polls)
    sleep = int(self.plan.params.get('sleep', 0)) if p3 else 0
    self.wfn = 'mbar_wait_s' if sleep else 'mbar_wait'
    lim = self.WAIT_NS if sleep else self.WAIT_LIMIT
    # which roles sleep: 1 all; 2 the epilogue and loader warps (the producers and the MMA
    # thread spin); 3 all but the MMA thread
    spin_roles = {2: ('mma', 'producers'), 3: ('mma',), 4: ('mma',)}.get(sleep, ())
    hybrid_roles = {4: ('producers',)}.get(sleep, ())

    def role(name):
      spin = name in spin_roles or not sleep
      self.wfn = 'mbar_wait' if spin else ('mbar_wait_h' if name in hybrid_roles else 'mbar_wait_s')
      return self.WAIT_LIMIT if spin else self.WAIT_NS
    # loader warp: 1 fetches all inputs of the next tile, 2 only the bulk copy of the B
    # blocks (the producers keep issuing the small R copies)
    self.loader_mode = int(self.plan.params.get('loader', 0)) if p3 else 0
    self.loader = self.loader_mode in (1, 2, 3, 4)
    nthreads = 32 * (4 * H + 1 + (4 if p3 else 0) + (1 if self.loader else 0))
    BAR_FULL, BAR_FREE, BAR_DFULL, BAR_DFREE = 0, nterms, 2 * nterms, 2 * nterms + 1
    if p3:
      # NS A slots used in turn by the terms (chunk c = it * terms + t takes slot c % NS),
      # ND accumulator pairs (tile it takes pair it % ND)
      self.NS = int(self.plan.params.get('slots', 2))
      self.ND = 1 if self.NS == nterms else 2
      self.dcols = 2 * n_mma
      self.scols = 2 * max(lay['a_cols'])
      self.d_base = self.NS * self.scols
      assert self.d_base + self.ND * self.dcols <= 512
      BAR_FULL, BAR_FREE = 0, self.NS
      BAR_DFULL, BAR_DFREE = 2 * self.NS, 2 * self.NS + self.ND
      self.BAR = dict(full=BAR_FULL, free=BAR_FREE, dfull=BAR_DFULL, dfree=BAR_DFREE,
                      stage=2 * self.NS + 2 * self.ND, sfree=2 * self.NS + 2 * self.ND + 1,
                      rstage=2 * self.NS + 2 * self.ND + 2)
      if self.direct:
        # two stage buffers, each with one barrier (bulk copy of B + the R scatter) and one
        # release barrier (the producers have read it)
        self.BAR['sfree'] = 2 * self.NS + 2 * self.ND + 2

    self.w(f'__global__ void __launch_bounds__({nthreads}, 1) {kname}({", ".join(self.params(globals_))}) {{')
    self.ind += 1
    self.w('extern __shared__ __align__(1024) unsigned char tfb_smem_raw[];')
    self.w(f'uint64_t* const bars = reinterpret_cast<uint64_t*>(tfb_smem_raw + {sm["off_bar"]});')
    nbars = ((2 * self.NS + 2 * self.ND + (4 if self.direct else 2 + (2 if self.rbuf2 else 0))) if p3
             else 2 * nterms + (3 if self.pipe == 2 else 2))
    BAR_STAGE = self.BAR['stage'] if p3 else 2 * nterms + 2
    self.w(f'unsigned* const tmem_slot = reinterpret_cast<unsigned*>(bars + {nbars});')
    probe_ns = int(self.plan.params.get('wait_probe_ns', 0))
    probe = int(self.plan.params.get('wait_probe', 0)) or probe_ns
    if probe:
      self.w(f'uint64_t* const probe_bar = bars + {nbars + 1};  // never arrived on')
      assert (nbars + 2) * 8 <= 256
    if self.direct:
      self.w(f'float* const stage = reinterpret_cast<float*>(tfb_smem_raw + {sm["off_stage"]});')
      self.w(f'float2* const sdp = reinterpret_cast<float2*>(tfb_smem_raw + {sm["off_sd"]});')
    elif self.pipe in (2, 3):
      self.w(f'float* const stage = reinterpret_cast<float*>(tfb_smem_raw + {sm["off_stage"]});')
      for ti in range(nterms):
        self.w(f'float* const ubuf{ti} = reinterpret_cast<float*>(tfb_smem_raw + {sm["off_u"] + ti * sm["ubuf_bytes"]});')
    else:
      self.w(f'float* const stage0 = reinterpret_cast<float*>(tfb_smem_raw + {sm["off_stage"]});')
      self.w(f'float* const stage1 = reinterpret_cast<float*>(tfb_smem_raw + {sm["off_stage"] + sm["stage"]});')
      self.w(f'float* const ubuf0 = reinterpret_cast<float*>(tfb_smem_raw + {sm["off_u"]});')
      self.w(f'float* const ubuf1 = reinterpret_cast<float*>(tfb_smem_raw + {sm["off_u"] + (sm["ubuf_bytes"] if sm["nbuf"] == 2 else 0)});')
    self.w('const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;')
    self.w(f'const size_t numTiles = (numElements + {te - 1}u) / {te}u;')
    # ---- setup: B operand, barriers, TMEM
    for ti, t in enumerate(s.terms):
      kp = lay['kpad'][ti]
      hi_off, lo_off = b_off[ti]
      sbo = (kp // ke) * 128
      self.open(f'for (int q = threadIdx.x; q < {rows_b * kp}; q += blockDim.x)')
      self.w(f'const int n = q / {kp}, k = q - n * {kp};')
      self.w(f'const int src = bgather{ti}_{b}[q];')
      self.w(f'const float v = src >= 0 ? {t.A.name}[src] : 0.0f;')
      self.w(f'const unsigned boff = (n >> 3) * {sbo}u + (k / {ke}) * 128u + (n & 7) * 16u + (k % {ke}) * {es}u;')
      if prec == 'tf32x3':
        self.w('unsigned hb, lb;')
        self.w('tfb_tc::tf32_split(v, hb, lb);')
        self.w(f'*reinterpret_cast<unsigned*>(tfb_smem_raw + {hi_off} + boff) = hb;')
        self.w(f'*reinterpret_cast<unsigned*>(tfb_smem_raw + {lo_off} + boff) = lb;')
      else:
        self.w('const __nv_bfloat16 h = __float2bfloat16_rn(v);')
        self.w('const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));')
        self.w(f'*reinterpret_cast<__nv_bfloat16*>(tfb_smem_raw + {hi_off} + boff) = h;')
        self.w(f'*reinterpret_cast<__nv_bfloat16*>(tfb_smem_raw + {lo_off} + boff) = l;')
      self.close()
    if self.direct:
      # the dense R pair buffers: zeros outside the patterns, written once
      self.open(f'for (int q = threadIdx.x; q < {2 * sm["sd_bytes"] // 16}; q += blockDim.x)')
      self.w('reinterpret_cast<float4*>(sdp)[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);')
      self.close()
    self.open('if (threadIdx.x == 0)')
    if p3:
      for i in range(self.NS):
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_FULL + i}], {NP}u);')
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_FREE + i}], 1u);')
      for i in range(self.ND):
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_DFULL + i}], 1u);')
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_DFREE + i}], 128u);')
      if self.loader and not self.direct:
        self.w(f'tfb_tc::mbar_init(&bars[{self.BAR["sfree"]}], 1u);')
    else:
      for ti in range(nterms):
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_FULL + ti}], {NP}u);')
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_FREE + ti}], 1u);')
      self.w(f'tfb_tc::mbar_init(&bars[{BAR_DFULL}], 1u);')
      self.w(f'tfb_tc::mbar_init(&bars[{BAR_DFREE}], {NP}u);')
    if self.direct:
      # per stage buffer: the B copy's arrival (bulk expect_tx, or lane 0 after the cp.async
      # fallback) + the 32 loader lanes' cp.async arrivals of the R scatter; its release
      # barrier counts the producer warps
      for i in range(2):
        self.w(f'tfb_tc::mbar_init(&bars[{BAR_STAGE + i}], 33u);')
        self.w(f'tfb_tc::mbar_init(&bars[{self.BAR["sfree"] + i}], {NP // 32}u);')
    elif self.pipe in (2, 3):
      # one arrival per copying thread (cp.async completion) + the bulk-copy issuer's expect_tx
      stage_count = {1: 32 + 1, 3: 1}.get(self.loader_mode, NP + 1)
      self.w(f'tfb_tc::mbar_init(&bars[{BAR_STAGE}], {stage_count}u);')
      if self.rbuf2:
        for i in range(2):
          self.w(f'tfb_tc::mbar_init(&bars[{self.BAR["rstage"] + i}], 32u);')
    if probe:
      self.w('tfb_tc::mbar_init(probe_bar, 1u);')
    self.w('asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");')
    self.close()
    self.open('if (warp == 0)')
    self.w('tfb_tc::tmem_alloc(tmem_slot, 512u);')
    self.close()
    self.w('tfb_tc::fence_proxy_async();')
    self.w('tfb_tc::fence_before();')
    self.w('__syncthreads();')
    self.w('tfb_tc::fence_after();')
    self.w('const unsigned tmem = *tmem_slot;')
    self.w('bool ok = true;')
    if probe:
      # nothing has been issued yet: on timeout every thread goes straight to the teardown
      if probe_ns:
        self.w(f'if (threadIdx.x == 0 && !tfb_tc::mbar_wait_s(probe_bar, 0u, {probe_ns}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 30u); }}')
      else:
        self.w(f'if (threadIdx.x == 0 && !tfb_tc::mbar_wait(probe_bar, 0u, {probe}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 30u); }}')
      self.w('ok = __syncthreads_and(ok ? 1 : 0) != 0;')
      self.open('if (ok)')
    # ---- MMA issuer
    if p3:
      self._mma_v3(s, lay, b_off, ke, es, idesc, role('mma'), n_mma)
    else:
      self.open(f'if (warp == {4 * H})')
      self.open('if (lane == 0)')
      self.w('unsigned it = 0;')
      self.open('for (size_t tile = blockIdx.x; tile < numTiles && ok; tile += gridDim.x, ++it)')
      self.w(f'if (it > 0 && !tfb_tc::{self.wfn}(&bars[{BAR_DFREE}], (it - 1u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 13u); break; }}')
      mma = 'mma_tf32' if prec == 'tf32x3' else 'mma_f16'
      for ti, t in enumerate(s.terms):
        kp = lay['kpad'][ti]
        ksteps = kp // lay['ks']
        hi_off, lo_off = b_off[ti]
        sbo = (kp // ke) * 128
        acols = lay['a_cols'][ti]
        cps = lay['ks'] * es // 4
        self.w(f'if (!tfb_tc::{self.wfn}(&bars[{BAR_FULL + ti}], it & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, {10 + ti}u); break; }}')
        self.w('tfb_tc::fence_after();')
        self.open(f'for (int ks = 0; ks < {ksteps}; ++ks)')
        self.w(f'const unsigned a_hi = tmem + {slot_base[ti]}u + ks * {cps}u;')
        self.w(f'const unsigned a_lo = a_hi + {acols}u;')
        self.w(f'const uint64_t bh = tfb_tc::smem_desc(tfb_tc::smem_u32(tfb_smem_raw + {hi_off}) + ks * 256u, 128u, {sbo}u);')
        self.w(f'const uint64_t bl = tfb_tc::smem_desc(tfb_tc::smem_u32(tfb_smem_raw + {lo_off}) + ks * 256u, 128u, {sbo}u);')
        first = '(ks > 0) ? 1u : 0u' if ti == 0 else '1u'
        self.w(f'tfb_tc::{mma}(tmem + {d_main}u, a_hi, bh, {idesc}u, {first});')
        self.w(f'tfb_tc::{mma}(tmem + {d_corr}u, a_hi, bl, {idesc}u, {first});')
        self.w(f'tfb_tc::{mma}(tmem + {d_corr}u, a_lo, bh, {idesc}u, 1u);')
        self.close()
        self.w(f'tfb_tc::mma_commit(&bars[{BAR_FREE + ti}]);')
      self.w(f'tfb_tc::mma_commit(&bars[{BAR_DFULL}]);')
      self.close()
      self.close()
      self.close()
    # ---- producers
    if p3 and self.direct:
      self._producers_direct(s, te, tcols, NP, lim, BAR_STAGE)
      self._epilogue_warps_v3(s, te, tcols, lim, n_mma)
      self._loader_direct(stage_off, lim, BAR_STAGE)
    elif p3:
      self._producers_v3(s, te, tcols, NP, stage_off, role('producers'), BAR_STAGE)
      self._epilogue_warps_v3(s, te, tcols, role('epilogue'), n_mma)
      if self.loader:
        self._loader_v3(stage_off, role('loader'), BAR_STAGE)
      role('rest')
    elif self.pipe == 2:
      self._producers_v2(s, te, tcols, NP, stage_off, slot_base, lim, BAR_DFULL, BAR_STAGE, d_main, d_corr)
    else:
      self.open(f'else if (warp < {4 * H})')
      self.w('const unsigned ptid = threadIdx.x;')
      self.w('const unsigned quad = warp & 3u, grp = warp >> 2;')
      self.w('const unsigned row = quad * 32u + lane;')
      self.w('const unsigned lane_addr = tmem + ((quad * 32u) << 16);')
      self.w(f'const bool lane_col = row < {tcols}u;')
      self.w(f'const unsigned le = row / {s.N}u, lj = row - le * {s.N}u;')
      self.w('unsigned it = 0;')
      self.w('size_t prev_tile = 0; bool have_prev = false;')
      self.open('if (blockIdx.x < numTiles)')
      self._prefetch('(size_t)blockIdx.x', 'stage0')
      self.close()
      self.w('tfb_tc::cp_async_commit();')
      self.open('for (size_t tile = blockIdx.x; ; tile += gridDim.x, ++it)')
      self.w('// every producer takes the same branches around named barriers: a timeout anywhere')
      self.w('// stops all producers at the next tile boundary (a barrier-wide OR), never mid-tile')
      self.w(f'if (tfb_tc::any_sync(1, {NP}, !ok)) break;')
      self.w('const bool more = tile < numTiles;')
      self.w('float* const cur = (it & 1u) ? stage1 : stage0;')
      self.w('float* const nxt = (it & 1u) ? stage0 : stage1;')
      self.open('if (more)')
      self.w('const size_t ntile = tile + gridDim.x;')
      self.open('if (ntile < numTiles)')
      self._prefetch('ntile', 'nxt')
      self.close()
      self.w('tfb_tc::cp_async_commit();')
      self.w('tfb_tc::cp_async_wait_one();')
      self.w(f'tfb_tc::named_sync(1, {NP});')
      self.w(f'const size_t e0 = tile * {te}u;')
      self.w('const size_t el = e0 + le;')
      self.w('const bool active = lane_col && el < numElements && (flags == nullptr || flags[el] != 0u);')
      for ti, t in enumerate(s.terms):
        self._term(ti, t, slot_base[ti], stage_off, lim, NP)
      self.close()
      # epilogue of the previous tile
      self.open('if (have_prev)')
      self.w(f'if (!tfb_tc::{self.wfn}(&bars[{BAR_DFULL}], (it - 1u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 20u); }}')
      self.w('tfb_tc::fence_after();')
      self._epilogue(d_main, d_corr, NP)
      self.close()
      self.w('if (!more) break;')
      self.w('prev_tile = tile; have_prev = true;')
      self.close()
      self.w('tfb_tc::cp_async_wait_all();')
      self.w('if (ptid == 0) tfb_tc::bulk_wait();')
      self.close()
    if probe:
      self.close()
    # ---- teardown
    self.w('tfb_tc::fence_before();')
    self.w('__syncthreads();')
    self.open('if (warp == 0)')
    self.w('tfb_tc::fence_after();')
    self.w('tfb_tc::tmem_dealloc(tmem, 512u);')
    self.close()
    self.ind -= 1
    self.w('}')
    kernel = '\n'.join(self.lines)
    args = []
    for t, _ in globals_:
      args.append(t.name)
      if t.addressing.name not in ('NONE', 'SCALAR'):
        args.append(f'{t.name}_extraOffset')
    args += ['numElements', 'flags']
    pre = ('  int sms = 0;\n'
           '  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);\n'
           '  if (sms > 0 && grid.x > (unsigned)sms) grid.x = (unsigned)sms;')
    launch = {'kernel': kname, 'block': nthreads, 'elements_per_block': te, 'smem': smem, 'args': args,
              'grid': f'(numElements + {te - 1}u) / {te}u', 'pre': pre}
    return kernel, launch, ''

  # ------------------------------------------------------------------ staging
  def _prefetch(self, tile_expr, buf):
    """cp.async the tile's batched operands into `buf` (16-byte chunks when aligned)."""
    te = self.sm['te']
    staged = staged_operands(self.s)
    NP = 128 * self.H
    off = 0
    for op, vals in staged:
      vp = _pad(vals, 4)
      self.open('')
      self.w(f'const size_t pe0 = ({tile_expr}) * {te}u;')
      if vals % 4 == 0:
        self.open(f'for (unsigned q = ptid; q < {te * vals // 4}u; q += {NP}u)')
        self.w(f'const unsigned ei = q / {vals // 4}u, c4 = q - ei * {vals // 4}u;')
        self.w('const size_t ee = pe0 + ei;')
        self.open('if (ee < numElements)')
        self.w(f'const float* src = {self._elem_ptr(op, "ee")} + 4u * c4;')
        self.w(f'float* dst = {buf} + {off} + ei * {vp}u + 4u * c4;')
        self.w('if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0u) tfb_tc::cp_async16(dst, src);')
        self.w('else { tfb_tc::cp_async4(dst, src); tfb_tc::cp_async4(dst + 1, src + 1); '
               'tfb_tc::cp_async4(dst + 2, src + 2); tfb_tc::cp_async4(dst + 3, src + 3); }')
        self.close()
        self.close()
      else:
        self.open(f'for (unsigned q = ptid; q < {te * vals}u; q += {NP}u)')
        self.w(f'const unsigned ei = q / {vals}u, c = q - ei * {vals}u;')
        self.w('const size_t ee = pe0 + ei;')
        self.w(f'if (ee < numElements) tfb_tc::cp_async4({buf} + {off} + ei * {vp}u + c, {self._elem_ptr(op, "ee")} + c);')
        self.close()
      self.close()
      off += te * vp

  # ------------------------------------------------------------------ one-pass pipeline
  def _cp_async_copy(self, op, vals, off, tile_expr, buf, NP):
    """cp.async one operand's values of a tile into `buf` + off (16-byte chunks when aligned)."""
    te = self.sm['te']
    vp = _pad(vals, 4)
    self.open('')
    self.w(f'const size_t pe0 = ({tile_expr}) * {te}u;')
    if op.addressing.name == 'PTR_BASED':
      # one element per warp at a time: its pointer is loaded once, not once per chunk
      self.open(f'for (unsigned ei = ptid >> 5; ei < {te}u; ei += {NP // 32}u)')
      self.w('const size_t ee = pe0 + ei;')
      self.w('if (ee >= numElements) break;')
      self.w(f'const float* const sbase = {self._elem_ptr(op, "ee")};')
      self.w(f'float* const dbase = {buf} + {off} + ei * {vp}u;')
      if vals % 4 == 0:
        self.w('const bool al = (reinterpret_cast<uintptr_t>(sbase) & 15u) == 0u;')
        self.open(f'for (unsigned c4 = ptid & 31u; c4 < {vals // 4}u; c4 += 32u)')
        self.w('const float* src = sbase + 4u * c4;')
        self.w('float* dst = dbase + 4u * c4;')
        self.w('if (al) tfb_tc::cp_async16(dst, src);')
        self.w('else { tfb_tc::cp_async4(dst, src); tfb_tc::cp_async4(dst + 1, src + 1); '
               'tfb_tc::cp_async4(dst + 2, src + 2); tfb_tc::cp_async4(dst + 3, src + 3); }')
        self.close()
      else:
        self.w(f'for (unsigned c = ptid & 31u; c < {vals}u; c += 32u) tfb_tc::cp_async4(dbase + c, sbase + c);')
      self.close()
      self.close()
      return
    if vals % 4 == 0:
      self.open(f'for (unsigned q = ptid; q < {te * vals // 4}u; q += {NP}u)')
      self.w(f'const unsigned ei = q / {vals // 4}u, c4 = q - ei * {vals // 4}u;')
      self.w('const size_t ee = pe0 + ei;')
      self.open('if (ee < numElements)')
      self.w(f'const float* src = {self._elem_ptr(op, "ee")} + 4u * c4;')
      self.w(f'float* dst = {buf} + {off} + ei * {vp}u + 4u * c4;')
      self.w('if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0u) tfb_tc::cp_async16(dst, src);')
      self.w('else { tfb_tc::cp_async4(dst, src); tfb_tc::cp_async4(dst + 1, src + 1); '
             'tfb_tc::cp_async4(dst + 2, src + 2); tfb_tc::cp_async4(dst + 3, src + 3); }')
      self.close()
      self.close()
    else:
      self.open(f'for (unsigned q = ptid; q < {te * vals}u; q += {NP}u)')
      self.w(f'const unsigned ei = q / {vals}u, c = q - ei * {vals}u;')
      self.w('const size_t ee = pe0 + ei;')
      self.w(f'if (ee < numElements) tfb_tc::cp_async4({buf} + {off} + ei * {vp}u + c, {self._elem_ptr(op, "ee")} + c);')
      self.close()
    self.close()

  def _loads_v2(self, tile_expr, part, stage_off, BAR_STAGE, NP, sync=True):
    """Inputs of tile `tile_expr` into the stage. part 1: the R blocks (cp.async by every
    producer; their region never overlaps the staged output). part 2: the B blocks, one
    bulk copy each when every block is contiguous and 16-byte aligned (issued by producer 0
    after its output bulk store has read the stage), else cp.async by every producer after
    a barrier; then every producer arrives on the stage barrier once its copies land."""
    sm = self.sm
    te = sm['te']
    if part == 1:
      for op in sm['r_ops']:
        vals = op.storage_size() if op.sparse else op.element_volume()
        self._cp_async_copy(op, vals, stage_off[op.name], tile_expr, 'stage', NP)
      return
    b_ops = sm['b_ops']
    eligible = all(_bulk_eligible(op, op.element_volume()) for op in b_ops)
    self.open('')
    self.w(f'const size_t be0 = ({tile_expr}) * {te}u;')
    self.w(f'const unsigned bnv = (unsigned)((numElements - be0) < {te}u ? (numElements - be0) : {te}u);')
    if eligible:
      conds = ' && '.join(f'((reinterpret_cast<uintptr_t>({op.name} + be0 * {op.element_volume()}u + '
                          f'{op.name}_extraOffset) & 15u) == 0u)' for op in b_ops)
      self.w(f'const bool bulk_in = {conds};')
    else:
      self.w('const bool bulk_in = false;')
    per_elem = sum(op.element_volume() * 4 for op in b_ops)
    self.open('if (bulk_in)')
    self.open('if (ptid == 0)')
    self.w(f'tfb_tc::mbar_arrive_expect_tx(&bars[{BAR_STAGE}], bnv * {per_elem}u);')
    for op in b_ops:
      self.w(f'tfb_tc::bulk_load(stage + {stage_off[op.name]}, {op.name} + be0 * {op.element_volume()}u + '
             f'{op.name}_extraOffset, bnv * {op.element_volume() * 4}u, &bars[{BAR_STAGE}]);')
    self.close()
    self.close()
    self.open('else')
    if sync:
      self.w(f'tfb_tc::named_sync(1, {NP});  // the previous tile\'s staged output has been read')
    for op in b_ops:
      self._cp_async_copy(op, op.element_volume(), stage_off[op.name], tile_expr, 'stage', NP)
    self.w(f'if (ptid == 0) tfb_tc::mbar_arrive(&bars[{BAR_STAGE}]);')
    self.close()
    self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
    self.close()

  def _u_phase_v2(self, stage_off, NP):
    """U_t = B * R_t for every term in one pass: one thread per (element, row l) loads row l
    of B once and writes row l of every U_t that uses it (R_t's pattern unrolled). With plan
    option `urows=2` a thread takes rows l and l + 1 (64-bit loads and stores, R's values
    loaded once for both)."""
    s, sm = self.s, self.sm
    te, pitch, N = sm['te'], sm['pitch'], s.N
    comp = ['x', 'y', 'z', 'w']
    two = int(self.plan.params.get('urows', 1)) == 2
    for B in sm['b_ops']:
      terms = [(ti, t) for ti, t in enumerate(s.terms) if t.B is B]
      K, P = terms[0][1].K, terms[0][1].P
      bvals = _pad(B.element_volume(), 4)
      ipe = K // 2 if two else K   # work items (rows or row pairs) per element
      if int(self.plan.params.get('uwarp', 0)) and ipe <= 32 and NP % 32 == 0:
        # warp-aligned items: a warp takes 32 // ipe whole elements (lanes past them idle),
        # so no warp's loads and stores straddle two elements' rows (one bank wavefront
        # fewer per access when ipe does not divide 32)
        epw = 32 // ipe
        self.w(f'const unsigned usub = lane / {ipe}u, uidx = lane - usub * {ipe}u;')
        self.open(f'for (unsigned ew = (ptid >> 5) * {epw}u + usub; ew < {_pad(te, epw)}u; ew += {NP // 32 * epw}u)')
        self.w(f'if (usub >= {epw}u || ew >= {te}u) continue;')
        self.w('const unsigned ei = ew;')
        self.w(f'const unsigned l = {"2u * uidx" if two else "uidx"};')
        if two:
          assert K % 2 == 0 and pitch % 2 == 0 and stage_off[B.name] % 2 == 0
        self.w(f'const float* const bq = stage + {stage_off[B.name]} + ei * {bvals}u + l;')
        for m in range(P):
          self.w(f'const float2 q{m} = *reinterpret_cast<const float2*>(bq + {m * K});' if two
                 else f'const float q{m} = bq[{m * K}];')
      elif two:
        assert K % 2 == 0 and pitch % 2 == 0 and stage_off[B.name] % 2 == 0
        self.open(f'for (unsigned q = ptid; q < {te * K // 2}u; q += {NP}u)')
        self.w(f'const unsigned ei = q / {K // 2}u, l = 2u * (q - ei * {K // 2}u);')
        self.w(f'const float* const bq = stage + {stage_off[B.name]} + ei * {bvals}u + l;')
        for m in range(P):
          self.w(f'const float2 q{m} = *reinterpret_cast<const float2*>(bq + {m * K});')
      else:
        self.open(f'for (unsigned q = ptid; q < {te * K}u; q += {NP}u)')
        self.w(f'const unsigned ei = q / {K}u, l = q - ei * {K}u;')
        self.w(f'const float* const bq = stage + {stage_off[B.name]} + ei * {bvals}u + l;')
        for m in range(P):
          self.w(f'const float q{m} = bq[{m * K}];')
      for ti, t in terms:
        dst = f'ubuf{ti}[(ei * {N}u + {{j}}u) * {pitch}u + l]'
        if t.R is None:
          for j in range(N):
            if two:
              self.w(f'*reinterpret_cast<float2*>(&{dst.format(j=j)}) = q{j};')
            else:
              self.w(f'{dst.format(j=j)} = q{j};')
          continue
        nr = t.R.storage_size()
        self.open('')
        rbase = 'rstage' if getattr(self, 'rbuf2', False) else 'stage'
        self.w(f'const float4* const rq = reinterpret_cast<const float4*>({rbase} + {stage_off[t.R.name]} + ei * {_pad(nr, 4)}u);')
        for v in range((nr + 3) // 4):
          self.w(f'const float4 r{v} = rq[{v}];')
        look = t.R.sparse_lookup() if t.R.sparse else None
        for j in range(N):
          ex, ey = '0.0f', '0.0f'
          for m in range(P):
            pos = look.get((m, j)) if look is not None else j * P + m
            if pos is not None:
              r = f'r{pos // 4}.{comp[pos % 4]}'
              if two:
                ex = f'fmaf(q{m}.x, {r}, {ex})'
                ey = f'fmaf(q{m}.y, {r}, {ey})'
              else:
                ex = f'fmaf(q{m}, {r}, {ex})'
          if two:
            self.w(f'*reinterpret_cast<float2*>(&{dst.format(j=j)}) = make_float2({ex}, {ey});')
          else:
            self.w(f'{dst.format(j=j)} = {ex};')
        self.close()
      self.close()

  def _producers_v2(self, s, te, tcols, NP, stage_off, slot_base, lim, BAR_DFULL, BAR_STAGE, d_main, d_corr):
    """Producer warps, one-pass pipeline. Per tile: [barrier D: abort OR] wait for the stage,
    U phase of all terms, [barrier A], R blocks of the next tile, epilogue of the previous
    tile ([barrier B] + bulk store when staged), B blocks of the next tile, lane phases."""
    b, H = self.base, self.H
    pitch = self.sm['pitch']
    self.open(f'else if (warp < {4 * H})')
    self.w('const unsigned ptid = threadIdx.x;')
    self.w('const unsigned quad = warp & 3u, grp = warp >> 2;')
    self.w('const unsigned row = quad * 32u + lane;')
    self.w('const unsigned lane_addr = tmem + ((quad * 32u) << 16);')
    self.w(f'const bool lane_col = row < {tcols}u;')
    self.w(f'const unsigned le = row / {s.N}u, lj = row - le * {s.N}u;')
    self.w('unsigned it = 0;')
    self.w('size_t prev_tile = 0; bool have_prev = false; bool pending = false;')
    self.open('if (blockIdx.x < numTiles)')
    self._loads_v2('(size_t)blockIdx.x', 1, stage_off, BAR_STAGE, NP)
    self._loads_v2('(size_t)blockIdx.x', 2, stage_off, BAR_STAGE, NP)
    self.w('pending = true;')
    self.close()
    self.open('for (size_t tile = blockIdx.x; ; tile += gridDim.x, ++it)')
    self.w('// every producer takes the same branches around named barriers: a timeout anywhere')
    self.w('// stops all producers at the next tile boundary (a barrier-wide OR), never mid-tile')
    self.w(f'if (tfb_tc::any_sync(1, {NP}, !ok)) break;')
    self.w('const bool more = tile < numTiles;')
    self.w('const size_t ntile = tile + gridDim.x;')
    self.w('const bool has_next = more && ntile < numTiles;')
    self.open('if (more)')
    self.w(f'if (!tfb_tc::{self.wfn}(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 40u); }}')
    self.w('pending = false;')
    self._u_phase_v2(stage_off, NP)
    self.close()
    self.w(f'tfb_tc::named_sync(1, {NP});')
    self.open('if (has_next)')
    self._loads_v2('ntile', 1, stage_off, BAR_STAGE, NP)
    self.close()
    self.open('if (have_prev)')
    self.w(f'if (!tfb_tc::{self.wfn}(&bars[{BAR_DFULL}], (it - 1u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 20u); }}')
    self.w('tfb_tc::fence_after();')
    self._epilogue(d_main, d_corr, NP, sbuf='stage', final_sync=False)
    self.close()
    self.open('if (has_next)')
    self._loads_v2('ntile', 2, stage_off, BAR_STAGE, NP)
    self.w('pending = true;')
    self.close()
    self.open('if (more)')
    self.w(f'const size_t e0 = tile * {te}u;')
    self.w('const size_t el = e0 + le;')
    self.w('const bool active = lane_col && el < numElements && (flags == nullptr || flags[el] != 0u);')
    # per term: the MMA thread starts on a term as soon as its slot is full
    if self.ahead and self._ahead_ok():
      self._lanes_ahead(slot_base, lim)
    else:
      for ti, t in enumerate(s.terms):
        self._lane(ti, t, slot_base[ti], lim, f'(ubuf{ti} + row * {pitch}u)', True)
    self.close()
    self.w('if (!more) break;')
    self.w('prev_tile = tile; have_prev = true;')
    self.close()
    self.w('// a stage load still in flight after an abort must land before the CTA exits')
    self.w(f'if (pending && !tfb_tc::{self.wfn}(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) atomicMax(&tfb_err_{b}, 41u);')
    self.w('tfb_tc::cp_async_wait_all();')
    self.w('if (ptid == 0) tfb_tc::bulk_wait();')
    self.close()

  # ------------------------------------------------------------------ warp-specialised pipeline
  # Barriers: FULL[NS] (A slot written, NP arrivals), FREE[NS] (A slot read by the MMAs, one
  # commit), DFULL[ND] (accumulator pair complete, one commit), DFREE[ND] (accumulator pair
  # read, 128 epilogue arrivals), STAGE (inputs landed), SFREE (stage consumed by the U pass,
  # for the loader warp). Term t of the CTA's it-th tile is chunk c = it * terms + t and uses
  # A slot c % NS (its (c / NS)-th use); tile it uses accumulator pair it % ND.
  def _mma_v3(self, s, lay, b_off, ke, es, idesc, lim, n_mma):
    b = self.base
    NS, ND, B = self.NS, self.ND, self.BAR
    mma = 'mma_tf32' if self.prec == 'tf32x3' else 'mma_f16'
    half = self.scols // 2
    self.open(f'if (warp == {4 * self.H})')
    self.open('if (lane == 0)')
    self.w('unsigned it = 0, chunk = 0;')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles && ok; tile += gridDim.x, ++it)')
    self.w(f'const unsigned db = it % {ND}u;')
    self.w(f'const unsigned d_main = tmem + {self.d_base}u + db * {self.dcols}u, d_corr = d_main + {n_mma}u;')
    self.w(f'if (it >= {ND}u && !tfb_tc::{self.wfn}(&bars[{B["dfree"]}u + db], ((it - {ND}u) / {ND}u) & 1u, {lim}ull)) '
           f'{{ ok = false; atomicMax(&tfb_err_{b}, 13u); break; }}')
    self.w('tfb_tc::fence_after();')
    for ti, t in enumerate(s.terms):
      kp = lay['kpad'][ti]
      ksteps = kp // lay['ks']
      hi_off, lo_off = b_off[ti]
      sbo = (kp // ke) * 128
      cps = lay['ks'] * es // 4
      self.w('{')
      self.w(f'const unsigned sl = chunk % {NS}u;')
      self.w(f'if (!tfb_tc::{self.wfn}(&bars[{B["full"]}u + sl], (chunk / {NS}u) & 1u, {lim}ull)) '
             f'{{ ok = false; atomicMax(&tfb_err_{b}, {10 + ti}u); break; }}')
      self.w('tfb_tc::fence_after();')
      first = '(ks > 0) ? 1u : 0u' if ti == 0 else '1u'
      idesc2 = (idesc & ~(0x3F << 17)) | (((2 * n_mma) >> 3) << 17)
      if self.fuse:
        # B rows [0, N) hi and [N, 2N) lo: one MMA writes main and correction side by side
        assert b_off[ti][1] - b_off[ti][0] == n_mma * kp * es
      # all products of a K step before the next step (grouping them by accumulator over the
      # K steps measured the same: 6.37e8 against 6.35e8 el/s)
      passes = ([('d_main', 'a_hi', 'bh', idesc2, first)] if self.fuse else
                [('d_main', 'a_hi', 'bh', idesc, first), ('d_corr', 'a_hi', 'bl', idesc, first)])
      passes.append(('d_corr', 'a_lo', 'bh', idesc, '1u'))
      for grp in [passes]:
        self.open(f'for (int ks = 0; ks < {ksteps}; ++ks)')
        self.w(f'const unsigned a_hi = tmem + sl * {self.scols}u + ks * {cps}u;')
        self.w(f'const unsigned a_lo = a_hi + {half}u;')
        self.w(f'const uint64_t bh = tfb_tc::smem_desc(tfb_tc::smem_u32(tfb_smem_raw + {hi_off}) + ks * 256u, 128u, {sbo}u);')
        if any(p[2] == 'bl' for p in grp):
          self.w(f'const uint64_t bl = tfb_tc::smem_desc(tfb_tc::smem_u32(tfb_smem_raw + {lo_off}) + ks * 256u, 128u, {sbo}u);')
        for d, a, bdesc, idv, acc in grp:
          self.w(f'tfb_tc::{mma}({d}, {a}, {bdesc}, {idv}u, {acc});')
        self.close()
      self.w(f'tfb_tc::mma_commit(&bars[{B["free"]}u + sl]);')
      self.w('++chunk;')
      self.w('}')
    self.w(f'tfb_tc::mma_commit(&bars[{B["dfull"]}u + db]);')
    self.close()
    self.close()
    self.close()

  def _lane_v3(self, ti, t, lim, src, nterms):
    """Lane phase of term ti into A slot (chunk % NS): wait until the MMAs of the chunk NS
    before have read the slot, split the lane's column of U_t and store hi / lo."""
    b = self.base
    NS, B = self.NS, self.BAR
    kp = self.lay['kpad'][ti]
    half = self.scols // 2
    self.open('')
    self.w(f'const unsigned chunk = it * {nterms}u + {ti}u, sl = chunk % {NS}u;')
    self.w(f'if (chunk >= {NS}u && !tfb_tc::{self.wfn}(&bars[{B["free"]}u + sl], ((chunk - {NS}u) / {NS}u) & 1u, {lim}ull)) '
           f'{{ ok = false; atomicMax(&tfb_err_{b}, {30 + ti}u); }}')
    self.w('tfb_tc::fence_after();')
    self.w(f'const unsigned slot = lane_addr + sl * {self.scols}u;')
    self.w('const unsigned c0 = grp * 16u;')
    self.open(f'if (c0 < {kp}u)')
    self.w('float u[16];')
    self.w('#pragma unroll')
    self.w('for (int i = 0; i < 16; ++i) u[i] = 0.0f;')
    self.open('if (active)')
    self.w(f'const float* p = {src} + c0;')
    if self.l64:
      for v in range(8):
        self.w(f'if (c0 + {2 * v}u < {t.K}u) {{ const float2 x = *reinterpret_cast<const float2*>(p + {2 * v}); '
               f'u[{2*v}] = x.x; u[{2*v+1}] = x.y; }}')
    else:
      for v in range(4):
        self.w(f'if (c0 + {4 * v}u < {t.K}u) {{ const float4 x = *reinterpret_cast<const float4*>(p + {4 * v}); '
               f'u[{4*v}] = x.x; u[{4*v+1}] = x.y; u[{4*v+2}] = x.z; u[{4*v+3}] = x.w; }}')
    self.close()
    self.w('unsigned hv[16], lv[16];')
    self.w('#pragma unroll')
    if int(self.plan.params.get('lpk', 0)):
      # lo = u - hi as packed FMAs (exact), 16 columns per tensor-memory store
      self.open('for (int p = 0; p < 8; ++p)')
      self.w('hv[2 * p] = tfb_tc::tf32_rna(u[2 * p]);')
      self.w('hv[2 * p + 1] = tfb_tc::tf32_rna(u[2 * p + 1]);')
      self.w('const float2 lo = __ffma2_rn(make_float2(__uint_as_float(hv[2 * p]), __uint_as_float(hv[2 * p + 1])), '
             'make_float2(-1.0f, -1.0f), make_float2(u[2 * p], u[2 * p + 1]));')
      self.w('lv[2 * p] = __float_as_uint(lo.x);')
      self.w('lv[2 * p + 1] = __float_as_uint(lo.y);')
      self.close()
      self.open(f'if (c0 + 8u < {kp}u)')
      self.w('tfb_tc::st_x16(slot + c0, hv);')
      self.w(f'tfb_tc::st_x16(slot + {half}u + c0, lv);')
      self.close()
      self.open('else')
      self.w('tfb_tc::st_x8(slot + c0, hv);')
      self.w(f'tfb_tc::st_x8(slot + {half}u + c0, lv);')
      self.close()
    else:
      self.w('for (int i = 0; i < 16; ++i) { hv[i] = tfb_tc::tf32_rna(u[i]); lv[i] = __float_as_uint(u[i] - __uint_as_float(hv[i])); }')
      self.w('tfb_tc::st_x8(slot + c0, hv);')
      self.w(f'tfb_tc::st_x8(slot + {half}u + c0, lv);')
      self.open(f'if (c0 + 8u < {kp}u)')
      self.w('tfb_tc::st_x8(slot + c0 + 8u, hv + 8);')
      self.w(f'tfb_tc::st_x8(slot + {half}u + c0 + 8u, lv + 8);')
      self.close()
    self.close()
    self.w('tfb_tc::st_wait();')
    self.w('tfb_tc::fence_before();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{B["full"]}u + sl]);')
    self.close()

  def _producers_v3(self, s, te, tcols, NP, stage_off, lim, BAR_STAGE):
    """Producer warps of the warp-specialised pipeline. Per tile: [barrier: abort OR] wait
    for the stage, U pass of all terms, [barrier], release the stage (to the loader warp, or
    issue the next tile's loads), lane phases of the terms into the A slots. The epilogue
    runs on its own warps."""
    b, H = self.base, self.H
    pitch = self.sm['pitch']
    nterms = len(s.terms)
    self.open(f'else if (warp < {4 * H})')
    self.w('const unsigned ptid = threadIdx.x;')
    self.w('const unsigned quad = warp & 3u, grp = warp >> 2;')
    self.w('const unsigned row = quad * 32u + lane;')
    self.w('const unsigned lane_addr = tmem + ((quad * 32u) << 16);')
    self.w(f'const bool lane_col = row < {tcols}u;')
    self.w(f'const unsigned le = row / {s.N}u;')
    self.w('unsigned it = 0;')
    if self.qreg:
      self._q_decl()
    rcopies = self.loader_mode not in (1, 3)   # the producers copy the R blocks
    if rcopies:
      self.w('bool pending = false;')
      self.open('if (blockIdx.x < numTiles)')
      self._loads_v2('(size_t)blockIdx.x', 1, stage_off, BAR_STAGE, NP)
      if self.loader_mode == 2:
        self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
      elif self.qreg:
        self._q_load('(size_t)blockIdx.x')
        self.w(f'if (ptid == 0) tfb_tc::mbar_arrive(&bars[{BAR_STAGE}]);')
        self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
      else:
        self._loads_v2('(size_t)blockIdx.x', 2, stage_off, BAR_STAGE, NP)
      self.w('pending = true;')
      self.close()
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it)')
    self.w('// every producer takes the same branches around named barriers: a timeout anywhere')
    self.w('// stops all producers at the next tile boundary (a barrier-wide OR), never mid-tile')
    self.w(f'if (tfb_tc::any_sync(1, {NP}, !ok)) break;')
    self.w(f'if (!tfb_tc::{self.wfn}(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, 40u); }}')
    if self.rbuf2:
      self.w(f'if (!tfb_tc::{self.wfn}(&bars[{self.BAR["rstage"]}u + (it & 1u)], (it >> 1) & 1u, {lim}ull)) '
             f'{{ ok = false; atomicMax(&tfb_err_{b}, 43u); }}')
      self.w(f'const float* const rstage = stage + ((it & 1u) ? {self.sm["rbuf_delta"]} : 0);')
    if rcopies:
      self.w('const size_t ntile = tile + gridDim.x;')
      self.w('const bool has_next = ntile < numTiles;')
      self.w('pending = false;')
    if self.qreg:
      self._u_phase_qreg(stage_off, NP)
      self.open('if (has_next)')
      self._q_load('ntile')   # in flight during this tile's lane phases
      self.close()
    else:
      self._u_phase_v2(stage_off, NP)
    self.w(f'tfb_tc::named_sync(1, {NP});')
    if self.loader:
      self.w(f'if (ptid == 0) tfb_tc::mbar_arrive(&bars[{self.BAR["sfree"]}]);  // the stage is free for the loader')
    if rcopies:
      self.open('if (has_next)')
      self._loads_v2('ntile', 1, stage_off, BAR_STAGE, NP)
      if self.loader_mode == 2:
        self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
      elif self.qreg:
        self.w(f'if (ptid == 0) tfb_tc::mbar_arrive(&bars[{BAR_STAGE}]);')
        self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{BAR_STAGE}]);')
      else:
        self._loads_v2('ntile', 2, stage_off, BAR_STAGE, NP)
      self.w('pending = true;')
      self.close()
    self.w(f'const size_t el = tile * {te}u + le;')
    self.w('const bool active = lane_col && el < numElements && (flags == nullptr || flags[el] != 0u);')
    for ti, t in enumerate(s.terms):
      self._lane_v3(ti, t, lim, f'(ubuf{ti} + row * {pitch}u)', nterms)
    self.close()
    if rcopies:
      self.w('// a stage load still in flight after an abort must land before the CTA exits')
      self.w(f'if (pending && !tfb_tc::{self.wfn}(&bars[{BAR_STAGE}], it & 1u, {lim}ull)) atomicMax(&tfb_err_{b}, 41u);')
      self.w('tfb_tc::cp_async_wait_all();')
      self.w('if (ptid == 0) tfb_tc::bulk_wait();')
    self.close()

  def _q_decl(self):
    """Registers holding this producer's two rows of the (single) B operand for one tile."""
    t0 = self.s.terms[0]
    self.w(f'float2 qv[{t0.P}];')
    self.w('#pragma unroll')
    self.w(f'for (int m = 0; m < {t0.P}; ++m) qv[m] = make_float2(0.0f, 0.0f);')

  def _q_load(self, tile_expr):
    """Rows l, l + 1 of B for producer item ptid of tile `tile_expr`, straight from global
    memory (64-bit loads when 8-byte aligned), zeros past the last element."""
    s = self.s
    t0 = s.terms[0]
    B, K, P = t0.B, t0.K, t0.P
    te = self.sm['te']
    self.open('')
    self.w(f'const unsigned ei = ptid / {K // 2}u, l = 2u * (ptid - ei * {K // 2}u);')
    self.w(f'const size_t e = ({tile_expr}) * {te}u + ei;')
    self.open(f'if (ptid < {te * K // 2}u && e < numElements)')
    self.w(f'const float* const src = {self._elem_ptr(B, "e")} + l;')
    self.open('if ((reinterpret_cast<uintptr_t>(src) & 7u) == 0u)')
    self.w('#pragma unroll')
    self.w(f'for (int m = 0; m < {P}; ++m) qv[m] = __ldg(reinterpret_cast<const float2*>(src + m * {K}));')
    self.close()
    self.open('else')
    self.w('#pragma unroll')
    self.w(f'for (int m = 0; m < {P}; ++m) qv[m] = make_float2(__ldg(src + m * {K}), __ldg(src + m * {K} + 1));')
    self.close()
    self.close()
    self.open('else')
    self.w('#pragma unroll')
    self.w(f'for (int m = 0; m < {P}; ++m) qv[m] = make_float2(0.0f, 0.0f);')
    self.close()
    self.close()

  def _u_phase_qreg(self, stage_off, NP):
    """U pass from the B rows in registers: producer ptid < te * K / 2 computes rows l, l + 1
    of every U_t (R_t from the stage, pattern unrolled) with 64-bit stores."""
    s, sm = self.s, self.sm
    te, pitch, N = sm['te'], sm['pitch'], s.N
    comp = ['x', 'y', 'z', 'w']
    K = s.terms[0].K
    self.open(f'if (ptid < {te * K // 2}u)')
    self.w(f'const unsigned ei = ptid / {K // 2}u, l = 2u * (ptid - ei * {K // 2}u);')
    for ti, t in enumerate(s.terms):
      dst = f'ubuf{ti}[(ei * {N}u + {{j}}u) * {pitch}u + l]'
      nr = t.R.storage_size()
      self.open('')
      self.w(f'const float4* const rq = reinterpret_cast<const float4*>(stage + {stage_off[t.R.name]} + ei * {_pad(nr, 4)}u);')
      for v in range((nr + 3) // 4):
        self.w(f'const float4 r{v} = rq[{v}];')
      look = t.R.sparse_lookup() if t.R.sparse else None
      for j in range(N):
        ex, ey = '0.0f', '0.0f'
        for m in range(t.P):
          pos = look.get((m, j)) if look is not None else j * t.P + m
          if pos is not None:
            r = f'r{pos // 4}.{comp[pos % 4]}'
            ex = f'fmaf(qv[{m}].x, {r}, {ex})'
            ey = f'fmaf(qv[{m}].y, {r}, {ey})'
        self.w(f'*reinterpret_cast<float2*>(&{dst.format(j=j)}) = make_float2({ex}, {ey});')
      self.close()
    self.close()

  def _bulk_b_only(self, tile_expr, stage_off, BAR_STAGE, dst='stage', bar=None):
    """Loader mode 2: the B blocks of a tile, one bulk copy by lane 0 with its expect_tx
    arrival; when a block is misaligned the 32 lanes copy it with cp.async, wait for their
    copies and lane 0 arrives (one arrival either way). `dst` and `bar` select another stage
    buffer and its barrier (loader mode 4)."""
    bar = bar if bar is not None else f'bars[{BAR_STAGE}]'
    sm = self.sm
    te = sm['te']
    b_ops = sm['b_ops']
    eligible = all(_bulk_eligible(op, op.element_volume()) for op in b_ops)
    self.open('')
    self.w(f'const size_t be0 = ({tile_expr}) * {te}u;')
    self.w(f'const unsigned bnv = (unsigned)((numElements - be0) < {te}u ? (numElements - be0) : {te}u);')
    if eligible:
      conds = ' && '.join(f'((reinterpret_cast<uintptr_t>({op.name} + be0 * {op.element_volume()}u + '
                          f'{op.name}_extraOffset) & 15u) == 0u)' for op in b_ops)
      self.w(f'const bool bulk_in = {conds};')
    else:
      self.w('const bool bulk_in = false;')
    per_elem = sum(op.element_volume() * 4 for op in b_ops)
    self.open('if (bulk_in)')
    self.open('if (lane == 0)')
    self.w(f'tfb_tc::mbar_arrive_expect_tx(&{bar}, bnv * {per_elem}u);')
    for op in b_ops:
      self.w(f'tfb_tc::bulk_load({dst} + {stage_off[op.name]}, {op.name} + be0 * {op.element_volume()}u + '
             f'{op.name}_extraOffset, bnv * {op.element_volume() * 4}u, &{bar});')
    self.close()
    self.close()
    self.open('else')
    for op in b_ops:
      self._cp_async_copy(op, op.element_volume(), stage_off[op.name], tile_expr, dst, 32)
    self.w('tfb_tc::cp_async_commit();  // wait_group only waits for committed copies')
    self.w('tfb_tc::cp_async_wait_all();')
    self.w('__syncwarp();')
    self.w(f'if (lane == 0) tfb_tc::mbar_arrive(&{bar});')
    self.close()
    self.close()

  def _r_copies(self, tile_expr, buf_expr, stage_off):
    """Loader mode 3: the R blocks of a tile into R buffer `buf_expr` (0 or 1) by the 32 lanes,
    each lane's copies counted on that buffer's mbarrier, then committed as one group."""
    self.open('')
    self.w(f'float* const rdst = stage + (({buf_expr}) ? {self.sm["rbuf_delta"]} : 0);')
    for op in self.sm['r_ops']:
      vals = op.storage_size() if op.sparse else op.element_volume()
      self._cp_async_copy(op, vals, stage_off[op.name], tile_expr, 'rdst', 32)
    self.w(f'tfb_tc::cp_async_mbar_arrive(&bars[{self.BAR["rstage"]}u + (({buf_expr}) ? 1u : 0u)]);')
    self.w('tfb_tc::cp_async_commit();')
    self.close()

  def _loader_v3(self, stage_off, lim, BAR_STAGE):
    """Loader warp: fetches the inputs of the next tile into the stage as soon as the
    producers have released it. Mode 1: B and R blocks; mode 2: the bulk copy of the B
    blocks only (the producers copy R); mode 3: the B blocks, and the R blocks one tile
    further ahead into two alternating R buffers, so the producers issue no copies."""
    b = self.base
    self.open('else')
    self.w('const unsigned ptid = lane;')
    self.w('unsigned it = 0;')
    self.w('bool pending = false;')
    if self.loader_mode == 3:
      self._r_copies('(size_t)blockIdx.x', '0u', stage_off)
      self.open('if ((size_t)blockIdx.x + gridDim.x < numTiles)')
      self._r_copies('(size_t)blockIdx.x + gridDim.x', '1u', stage_off)
      self.close()
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it)')
    self.w(f'if (it > 0u && !tfb_tc::{self.wfn}(&bars[{self.BAR["sfree"]}], (it - 1u) & 1u, {lim}ull)) '
           f'{{ ok = false; atomicMax(&tfb_err_{b}, 42u); break; }}')
    if self.loader_mode == 1:
      self._loads_v2('tile', 1, stage_off, BAR_STAGE, 32)
      self._loads_v2('tile', 2, stage_off, BAR_STAGE, 32, sync=False)
    else:
      self._bulk_b_only('tile', stage_off, BAR_STAGE)
    if self.loader_mode == 3:
      # R of tile it + 1 into the buffer tile it - 1 has released
      self.open('if (it > 0u && tile + gridDim.x < numTiles)')
      self._r_copies('tile + gridDim.x', '(it + 1u) & 1u', stage_off)
      self.close()
    self.w('pending = true;')
    self.close()
    self.w('// copies still in flight must land before the CTA exits: the last tile\'s, consumed')
    self.w('// by the producers, or one nobody consumed after an abort')
    self.w(f'if (pending && !tfb_tc::{self.wfn}(&bars[{BAR_STAGE}], (it - 1u) & 1u, {lim}ull)) atomicMax(&tfb_err_{b}, 41u);')
    self.w('tfb_tc::cp_async_wait_all();')
    self.w('if (lane == 0) tfb_tc::bulk_wait();')
    self.close()

  def _sd_slots(self):
    """(term, storage position) pairs of the R factors in scatter order, with each one's pair
    index (t * P + m) * 128 + j in the dense pair buffer (the element adds e * N)."""
    s = self.s
    P, N = s.terms[0].P, s.N
    slots = []
    for ti, t in enumerate(s.terms):
      R = t.R
      if R.sparse:
        look = R.sparse_lookup()
        inv = {pos: mj for mj, pos in look.items()}
        nv = R.storage_size()
      else:
        inv = {j * P + m: (m, j) for m in range(P) for j in range(N)}
        nv = P * N
      for pos in range(nv):
        m, j = inv[pos]
        slots.append((ti, pos, (ti * P + m) * 128 + j))
    return slots

  def _sd_table_decl(self):
    """File-scope table of the loader lanes' R scatter slots: one packed word per slot, pair
    index + 1 (0: no slot) in bits 0-15, term in bits 16-23, storage position in 24-31."""
    slots = self._sd_slots()
    nsl = len(slots)
    kq = (nsl + 31) // 32
    assert all(sl[2] + 1 < (1 << 16) and sl[1] < 256 for sl in slots)
    words = [((d + 1) | (ti << 16) | (pos << 24)) for ti, pos, d in slots] + [0] * (32 * kq - nsl)
    self.sd_kq = kq
    self.w(f'__device__ const unsigned sdslot_{self.base}[{32 * kq}] = {{{", ".join(f"{w_}u" for w_ in words)}}};')

  def _producers_direct(self, s, te, tcols, NP, lim, BAR_STAGE):
    """Direct-lane producers: producer (quadrant, group) owns TMEM lane row = flat column
    c = e * N + j of the tile and the K columns [16 grp, 16 grp + 16). Per tile: wait for the
    stage buffer, compute U_t[l, c] = sum_m B_e[l, m] R_t[m, j] for its K columns and every
    term (m ascending, packed FMAs over two rows with the dense R pair (R, R); zeros outside
    R's pattern), release the stage, then per term split into TF32 hi / lo and store them to
    that term's A slot."""
    b, H = self.base, self.H
    sm = self.sm
    nterms = len(s.terms)
    t0 = s.terms[0]
    K, P, N = t0.K, t0.P, s.N
    kp = self.lay['kpad'][0]
    half = self.scols // 2
    NS, BR = self.NS, self.BAR
    bvals = sm['bvals']
    self.open(f'else if (warp < {4 * H})')
    self.w('const unsigned quad = warp & 3u, grp = warp >> 2;')
    self.w('const unsigned row = quad * 32u + lane;')
    self.w('const unsigned lane_addr = tmem + ((quad * 32u) << 16);')
    self.w(f'const bool lane_col = row < {tcols}u;')
    self.w(f'const unsigned le = row / {N}u;')
    self.w(f'const unsigned lec = le < {te}u ? le : {te - 1}u;  // in-bounds stage reads for the padding lanes')
    self.w('const unsigned c0 = grp * 16u;')
    self.w('const float2 neg1 = make_float2(-1.0f, -1.0f);')
    self.w('unsigned it = 0;')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it)')
    self.w('// every producer takes the same branches around the barrier: a timeout anywhere stops')
    self.w('// all producers at the next tile boundary (a barrier-wide OR), never mid-tile')
    self.w(f'if (tfb_tc::any_sync(1, {NP}, !ok)) break;')
    self.w('const unsigned sb = it & 1u;')
    self.w(f'if (!tfb_tc::{self.wfn}(&bars[{BAR_STAGE}u + sb], (it >> 1) & 1u, {lim}ull)) '
           f'{{ ok = false; atomicMax(&tfb_err_{b}, 40u); }}')
    self.w(f'const float* const qs = stage + (sb ? {sm["sdelta"]}u : 0u) + lec * {bvals}u + c0;')
    self.w(f'const float2* const sd = sdp + (sb ? {sm["sd_delta"]}u : 0u) + row;')
    self.w(f'float2 acc[{nterms}][8];')
    self.w(f'for (int t = 0; t < {nterms}; ++t) for (int p = 0; p < 8; ++p) acc[t][p] = make_float2(0.0f, 0.0f);')
    # full groups (16 columns) and the last, partial group
    ncols_list = sorted({min(16, K - 16 * g) for g in range(H) if K - 16 * g > 0}, reverse=True)
    for idx, ncols in enumerate(ncols_list):
      if len(ncols_list) == 1:
        self.open(f'if (c0 < {K}u)')
      elif idx == 0:
        self.open(f'if (c0 + {ncols}u <= {K}u)')
      else:
        self.open(f'else if (c0 < {K}u)')
      nv4 = ncols // 4
      for m in range(P):
        self.open('')
        for ti in range(nterms):
          self.w(f'const float2 s{ti} = sd[{(ti * P + m) * 128}];')
        # the row in halves of 8 columns: fewer live registers, the same loads
        for h0 in range(0, nv4, 2):
          self.open('')
          for v in range(h0, min(nv4, h0 + 2)):
            self.w(f'const float4 x{v} = *reinterpret_cast<const float4*>(qs + {m * K + 4 * v});')
          for ti in range(nterms):
            for v in range(h0, min(nv4, h0 + 2)):
              self.w(f'acc[{ti}][{2 * v}] = __ffma2_rn(make_float2(x{v}.x, x{v}.y), s{ti}, acc[{ti}][{2 * v}]);')
              self.w(f'acc[{ti}][{2 * v + 1}] = __ffma2_rn(make_float2(x{v}.z, x{v}.w), s{ti}, acc[{ti}][{2 * v + 1}]);')
          self.close()
        self.close()
      self.close()
    self.w('__syncwarp();')
    self.w(f'if (lane == 0) tfb_tc::mbar_arrive(&bars[{BR["sfree"]}u + sb]);  // this warp has read the stage buffer')
    self.w(f'const size_t el = tile * {te}u + le;')
    self.w('const bool active = lane_col && el < numElements && (flags == nullptr || flags[el] != 0u);')
    for ti in range(nterms):
      self.open('')
      self.w(f'const unsigned chunk = it * {nterms}u + {ti}u, sl = chunk % {NS}u;')
      self.w(f'if (chunk >= {NS}u && !tfb_tc::{self.wfn}(&bars[{BR["free"]}u + sl], ((chunk - {NS}u) / {NS}u) & 1u, {lim}ull)) '
             f'{{ ok = false; atomicMax(&tfb_err_{b}, {30 + ti}u); }}')
      self.w('tfb_tc::fence_after();')
      self.w(f'const unsigned slot = lane_addr + sl * {self.scols}u;')
      self.open(f'if (c0 < {kp}u)')
      self.w('unsigned hv[16], lv[16];')
      self.w('#pragma unroll')
      self.open('for (int p = 0; p < 8; ++p)')
      self.w(f'const float2 u = active ? acc[{ti}][p] : make_float2(0.0f, 0.0f);')
      self.w('hv[2 * p] = tfb_tc::tf32_rna(u.x);')
      self.w('hv[2 * p + 1] = tfb_tc::tf32_rna(u.y);')
      self.w('const float2 lo = __ffma2_rn(make_float2(__uint_as_float(hv[2 * p]), __uint_as_float(hv[2 * p + 1])), neg1, u);')
      self.w('lv[2 * p] = __float_as_uint(lo.x);')
      self.w('lv[2 * p + 1] = __float_as_uint(lo.y);')
      self.close()
      self.w('tfb_tc::st_x8(slot + c0, hv);')
      self.w(f'tfb_tc::st_x8(slot + {half}u + c0, lv);')
      self.open(f'if (c0 + 8u < {kp}u)')
      self.w('tfb_tc::st_x8(slot + c0 + 8u, hv + 8);')
      self.w(f'tfb_tc::st_x8(slot + {half}u + c0 + 8u, lv + 8);')
      self.close()
      self.close()
      self.w('tfb_tc::st_wait();')
      self.w('tfb_tc::fence_before();')
      self.w(f'tfb_tc::mbar_arrive(&bars[{BR["full"]}u + sl]);')
      self.close()
    self.close()
    self.close()

  def _loader_direct(self, stage_off, lim, BAR_STAGE):
    """Loader mode 4 (direct-lane producers): tiles it and it + 1 in flight in two stage
    buffers. Once the producers have released buffer it & 1 (its own release barrier, so a
    release two tiles ahead cannot alias), the warp fills it with tile it + 2: the bulk copy
    of the B blocks, and the R values scattered as (R, R) pairs into the dense pair buffer
    by 4-byte cp.async copies (lane q takes the (term, position) slots q, q + 32, ... of
    every element), each lane's copies counted on the buffer's barrier."""
    b = self.base
    sm = self.sm
    te, N = sm['te'], self.s.N
    kq = self.sd_kq
    self.open('else')
    self.w('const unsigned ptid = lane;')
    for k in range(kq):
      self.w(f'const unsigned sw{k} = sdslot_{b}[{32 * k}u + lane];')
      self.w(f'const int sdst{k} = (int)(sw{k} & 0xFFFFu) - 1;')
      self.w(f'const unsigned sterm{k} = (sw{k} >> 16) & 0xFFu, spos{k} = sw{k} >> 24;')
    r_of_term = [t.R for t in self.s.terms]
    ptr_based = [R.addressing.name == 'PTR_BASED' for R in r_of_term]
    # per slot, once per CTA: the R operand's base (strided: the first element's value at
    # the slot's position; pointer arrays: the pointer table, the position added per element)
    for k in range(kq):
      if any(ptr_based):
        self.w(f'const float* const* sptab{k} = nullptr; unsigned soff{k} = 0u;')
      self.w(f'const float* sbase{k} = nullptr; unsigned svol{k} = 0u;')
      for ti, R in enumerate(r_of_term):
        self.open(f'{"if" if ti == 0 else "else if"} (sterm{k} == {ti}u)')
        if ptr_based[ti]:
          self.w(f'sptab{k} = {R.name}; soff{k} = {R.name}_extraOffset + spos{k};')
        else:
          self.w(f'sbase{k} = {R.name} + {R.name}_extraOffset + spos{k}; svol{k} = {R.element_volume()}u;')
        self.close()

    def src_expr(k, e):
      if not any(ptr_based):
        return f'sbase{k} + ({e}) * svol{k}'
      if all(ptr_based):
        return f'sptab{k}[{e}] + soff{k}'
      return f'(sptab{k} != nullptr ? sptab{k}[{e}] + soff{k} : sbase{k} + ({e}) * svol{k})'

    def fill(tile_expr, buf_expr):
      bar = f'bars[{BAR_STAGE}u + (({buf_expr}) ? 1u : 0u)]'
      self._bulk_b_only(tile_expr, stage_off, BAR_STAGE, dst=f'(stage + (({buf_expr}) ? {sm["sdelta"]}u : 0u))', bar=bar)
      self.open('')
      self.w(f'float* const sdf = reinterpret_cast<float*>(sdp + (({buf_expr}) ? {sm["sd_delta"]}u : 0u));')
      self.w(f'const size_t fe0 = ({tile_expr}) * {te}u;')
      self.w(f'const unsigned fnv = (unsigned)((numElements - fe0) < {te}u ? (numElements - fe0) : {te}u);')
      self.w('#pragma unroll 2')
      self.open('for (unsigned ei = 0; ei < fnv; ++ei)')
      for k in range(kq):
        self.open(f'if (sdst{k} >= 0)')
        self.w(f'const float* const src = {src_expr(k, "fe0 + ei")};')
        self.w(f'float* const dst = sdf + 2u * ((unsigned)sdst{k} + ei * {N}u);')
        self.w('tfb_tc::cp_async4(dst, src);')
        self.w('tfb_tc::cp_async4(dst + 1, src);')
        self.close()
      self.close()
      self.w(f'tfb_tc::cp_async_mbar_arrive(&{bar});')
      self.w('tfb_tc::cp_async_commit();')
      self.close()

    self.w('unsigned nis0 = 0, nis1 = 0;  // fills issued into each buffer')
    self.open('if ((size_t)blockIdx.x < numTiles)')
    fill('(size_t)blockIdx.x', '0u')
    self.w('++nis0;')
    self.close()
    self.open('if ((size_t)blockIdx.x + gridDim.x < numTiles)')
    fill('(size_t)blockIdx.x + gridDim.x', '1u')
    self.w('++nis1;')
    self.close()
    self.w('unsigned it = 0;')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it)')
    self.w('const size_t nt = tile + 2u * (size_t)gridDim.x;')
    self.w('if (nt >= numTiles) continue;')
    self.w(f'if (!tfb_tc::{self.wfn}(&bars[{self.BAR["sfree"]}u + (it & 1u)], (it >> 1) & 1u, {lim}ull)) '
           f'{{ ok = false; atomicMax(&tfb_err_{b}, 42u); break; }}')
    fill('nt', 'it & 1u')
    self.w('if (it & 1u) ++nis1; else ++nis0;')
    self.close()
    self.w('// fills still in flight must land before the CTA exits (consumed, or not after an abort)')
    self.w(f'if (nis0 && !tfb_tc::{self.wfn}(&bars[{BAR_STAGE}], (nis0 - 1u) & 1u, {lim}ull)) atomicMax(&tfb_err_{b}, 41u);')
    self.w(f'if (nis1 && !tfb_tc::{self.wfn}(&bars[{BAR_STAGE + 1}], (nis1 - 1u) & 1u, {lim}ull)) atomicMax(&tfb_err_{b}, 41u);')
    self.w('tfb_tc::cp_async_wait_all();')
    self.close()

  def _epilogue_warps_v3(self, s, te, tcols, lim, n_mma):
    """Four epilogue warps (one per TMEM lane quadrant): per tile, wait for the accumulator
    pair, read it (main + correction), release it to the MMAs and store the lane's output
    column straight to global memory (16-byte stores when aligned)."""
    b = self.base
    M = s.M
    out = s.out
    nld = (M + 7) // 8
    self.open(f'else if (warp < {4 * self.H + 5})' if self.loader else 'else')
    self.w('const unsigned equad = warp & 3u;')
    self.w('const unsigned erow = equad * 32u + lane;')
    self.w('const unsigned e_addr = tmem + ((equad * 32u) << 16);')
    self.w(f'const bool ecol = erow < {tcols}u;')
    self.w(f'const unsigned ele = erow / {s.N}u, elj = erow - ele * {s.N}u;')
    self.w('unsigned it = 0;')
    self.open('for (size_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it)')
    self.w(f'const unsigned db = it % {self.ND}u;')
    self.w(f'if (!tfb_tc::{self.wfn}(&bars[{self.BAR["dfull"]}u + db], (it / {self.ND}u) & 1u, {lim}ull)) '
           f'{{ ok = false; atomicMax(&tfb_err_{b}, 20u); break; }}')
    self.w('tfb_tc::fence_after();')
    self.w(f'const unsigned dm = e_addr + {self.d_base}u + db * {self.dcols}u;')
    estg = (self.estg and out.addressing.name == 'STRIDED' and not s.accumulate
            and out.element_volume() == M * s.N and M % 8 == 0)
    if estg:
      # 16x256b reads: each group of 4 threads holds 8 consecutive values of one output
      # column, so every warp store writes whole 32-byte sectors (no staging buffer)
      vol = out.element_volume()
      self.w(f'float* const obase = {out.name} + tile * {te * vol}u + {out.name}_extraOffset;')
      self.open('if (flags == nullptr && (reinterpret_cast<uintptr_t>(obase) & 7u) == 0u)')
      self.w(f'float ev[{2 * nld * 4}];')
      for h in range(2):
        for k0 in range(0, nld, 2):
          ks = list(range(k0, min(nld, k0 + 2)))
          self.open('')
          self.w(f'unsigned dv[{4 * len(ks)}], dc[{4 * len(ks)}];')
          for i, k in enumerate(ks):
            self.w(f'tfb_tc::ld16x256(dm + {(16 * h) << 16}u + {8 * k}u, dv + {4 * i});')
            self.w(f'tfb_tc::ld16x256(dm + {(16 * h) << 16}u + {n_mma + 8 * k}u, dc + {4 * i});')
          self.w('tfb_tc::ld_wait();')
          self.w('#pragma unroll')
          self.w(f'for (int i = 0; i < {4 * len(ks)}; ++i) ev[{(h * nld + k0) * 4} + i] = __uint_as_float(dv[i]) + __uint_as_float(dc[i]);')
          self.close()
      self.w('tfb_tc::fence_before();')
      self.w(f'tfb_tc::mbar_arrive(&bars[{self.BAR["dfree"]}u + db]);')
      self.w(f'const size_t nrows = (numElements - tile * {te}u) < {te}u ? (numElements - tile * {te}u) * {s.N}u : {te * s.N}u;')
      self.w('const unsigned er = equad * 32u + (lane >> 2), ew = 2u * (lane & 3u);')
      for h in range(2):
        for half in range(2):
          c = f'er + {16 * h + 8 * half}u'
          self.open(f'if ({c} < nrows)')
          self.w(f'float* const ocol = obase + (size_t)({c}) * {M}u + ew;')
          for k in range(nld):
            base = (h * nld + k) * 4 + 2 * half
            self.w(f'*reinterpret_cast<float2*>(ocol + {8 * k}) = make_float2(ev[{base}], ev[{base + 1}]);')
          self.close()
      self.close()
      self.open('else')
    self.w(f'float acc[{nld * 8}];')
    for k0 in range(0, nld, 2):
      ks = list(range(k0, min(nld, k0 + 2)))
      self.open('')
      self.w(f'unsigned dv[{8 * len(ks)}], dc[{8 * len(ks)}];')
      for i, k in enumerate(ks):
        self.w(f'tfb_tc::ld_x8(dm + {8 * k}u, dv + {8 * i});')
        self.w(f'tfb_tc::ld_x8(dm + {n_mma + 8 * k}u, dc + {8 * i});')
      self.w('tfb_tc::ld_wait();')
      self.w('#pragma unroll')
      if int(self.plan.params.get('epk', 0)):
        self.w(f'for (int i = 0; i < {4 * len(ks)}; ++i) {{ const float2 v = __fadd2_rn('
               'make_float2(__uint_as_float(dv[2 * i]), __uint_as_float(dv[2 * i + 1])), '
               'make_float2(__uint_as_float(dc[2 * i]), __uint_as_float(dc[2 * i + 1]))); '
               f'acc[{8 * k0} + 2 * i] = v.x; acc[{8 * k0} + 2 * i + 1] = v.y; }}')
      else:
        self.w(f'for (int i = 0; i < {8 * len(ks)}; ++i) acc[{8 * k0} + i] = __uint_as_float(dv[i]) + __uint_as_float(dc[i]);')
      self.close()
    self.w('tfb_tc::fence_before();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{self.BAR["dfree"]}u + db]);')
    self.w(f'const size_t pel = tile * {te}u + ele;')
    staged = ('off_ost' in self.sm and out.addressing.name == 'STRIDED' and not s.accumulate
              and out.element_volume() == M * s.N and M % 4 == 0 and int(self.plan.params.get('ostage', 1))
              and not estg)
    if staged:
      # the warp's 32 rows are 32 consecutive output columns of the tile: stage them in
      # shared memory and write them with one bulk copy (unmasked, 16-byte aligned output)
      vol = out.element_volume()
      self.w(f'float* const obase = {out.name} + tile * {te * vol}u + {out.name}_extraOffset;')
      self.open('if (flags == nullptr && (reinterpret_cast<uintptr_t>(obase) & 15u) == 0u)')
      self.w(f'float* const ost = reinterpret_cast<float*>(tfb_smem_raw + {self.sm["off_ost"]});')
      orows = self.sm['ost_rows']
      self.w(f'const size_t nrows = (numElements - tile * {te}u) < {te}u ? (numElements - tile * {te}u) * {s.N}u : {te * s.N}u;')
      swz = self.oswz and not self.opad and (M // 4) % 2 == 0
      if swz:
        # rows 4r..4r+3 with r odd write each pair of 16-byte chunks in swapped order: the 8
        # rows of a store phase then fall on 8 distinct bank groups (a row is 14 chunks)
        self.w('const unsigned sw = (lane >> 2) & 1u;')
        self.w('#pragma unroll')
        self.open(f'for (int i = 0; i < {M // 4}; i += 2)')
        self.w('#pragma unroll')
        self.w('for (int q = 0; q < 4; ++q) { const float t = acc[4 * i + q]; '
               'acc[4 * i + q] = sw ? acc[4 * i + 4 + q] : t; acc[4 * i + 4 + q] = sw ? t : acc[4 * i + 4 + q]; }')
        self.close()
      if self.opad:
        # padded rows (pitch M + 4 floats): each lane stages its row and issues its own bulk
        # copy; a lane waits for its own earlier copies, and the warp syncs before another
        # half of the lanes reuses the rows
        OP = self.sm['ost_pitch']
        for h in range(32 // orows):
          self.w(f'{"if (it > 0) " if h == 0 else ""}tfb_tc::bulk_wait_read();  // this lane\'s earlier copies have read the buffer')
          self.w('__syncwarp();')
          self.open(f'if (ecol && (lane / {orows}u) == {h}u)')
          self.w(f'float* const orow = ost + (equad * {orows}u + (lane - {h * orows}u)) * {OP}u;')
          self.w('#pragma unroll')
          self.w(f'for (int i = 0; i < {M // 4}; ++i) reinterpret_cast<float4*>(orow)[i] = '
                 'make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);')
          self.w('tfb_tc::fence_proxy_async();')
          self.w('const size_t r = equad * 32u + lane;')
          self.w(f'if (r < nrows) tfb_tc::bulk_store(obase + r * {M}u, orow, {M * 4}u);')
          self.close()
      for h in range(32 // orows if not self.opad else 0):
        # rows [r0, r0 + orows) of the warp go through its buffer of orows rows
        self.w(f'if (lane == 0 && (it > 0{" || true" if h else ""})) tfb_tc::bulk_wait_read();  // the buffer\'s previous copy has read it')
        self.w('__syncwarp();')
        self.w('// rows past the tile\'s columns have no place in the buffer')
        self.open(f'if (ecol && (lane / {orows}u) == {h}u)')
        self.w(f'float* const orow = ost + (equad * {orows}u + (lane - {h * orows}u)) * {M}u;')
        if swz:
          self.w('#pragma unroll')
          self.w(f'for (int i = 0; i < {M // 4}; ++i) reinterpret_cast<float4*>(orow)[i ^ sw] = '
                 'make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);')
        else:
          self.w('#pragma unroll')
          self.w(f'for (int i = 0; i < {M // 4}; ++i) reinterpret_cast<float4*>(orow)[i] = '
                 'make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);')
        self.close()
        self.w('tfb_tc::fence_proxy_async();')
        self.w('__syncwarp();')
        self.open('if (lane == 0)')
        self.w(f'const size_t r0 = equad * 32u + {h * orows}u;')
        self.w(f'const unsigned rows = nrows > r0 ? (unsigned)(nrows - r0 < {orows}u ? nrows - r0 : {orows}u) : 0u;')
        self.w(f'if (rows > 0u) tfb_tc::bulk_store(obase + r0 * {M}u, ost + equad * {orows * M}u, rows * {M * 4}u);')
        self.close()
      self.close()
      self.open('else if (ecol && pel < numElements && (flags == nullptr || flags[pel] != 0u))')
    else:
      self.open('if (ecol && pel < numElements && (flags == nullptr || flags[pel] != 0u))')
    self.w(f'float* const col = {self._elem_ptr(out, "pel")} + (size_t)elj * {M}u;')
    if M % 4 == 0 and not s.accumulate:
      self.open('if ((reinterpret_cast<uintptr_t>(col) & 15u) == 0u)')
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {M // 4}; ++i) reinterpret_cast<float4*>(col)[i] = '
             'make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);')
      self.close()
      self.open('else')
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {M}; ++i) col[i] = acc[i];')
      self.close()
    elif s.accumulate:
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {M}; ++i) col[i] += acc[i];')
    else:
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {M}; ++i) col[i] = acc[i];')
    self.close()
    if estg:
      self.close()   # the else branch of the sector-store path
    self.close()
    if staged:
      self.w(f'{"" if self.opad else "if (lane == 0) "}tfb_tc::bulk_wait();  // the last bulk stores have landed')
    self.close()

  # ------------------------------------------------------------------ producer
  def _term(self, ti, t, slot_col, stage_off, lim, NP):
    b, LC = self.base, self.LC
    s = self.s
    lay = self.lay
    prec = self.prec
    kp = lay['kpad'][ti]
    acols = lay['a_cols'][ti]
    nterms = len(s.terms)
    pitch = self.sm['pitch']
    te = self.sm['te']
    H = self.H
    bvals = _pad(t.B.element_volume(), 4)
    self.w(f'// term {ti}: U_{ti} -> tensor memory slot {ti} (hi at +0, lo at +{acols})')
    self.open('')
    ubuf = f'ubuf{ti % self.sm["nbuf"]}' if self.sm['nbuf'] == 2 else 'ubuf0'
    if t.R is not None:
      # U phase: thread (element group g = ptid / KP2, row l = ptid % KP2) computes row l of
      # U_t for every column j of elements g, g + NP/KP2, ... (no integer division)
      rvals = _pad(t.R.storage_size(), 4)
      kp2 = 1
      while kp2 < t.K:
        kp2 *= 2
      groups = max(1, NP // kp2)
      self.w(f'const unsigned l = ptid & {kp2 - 1}u, g = ptid / {kp2}u;')
      self.open(f'if (l < {t.K}u)')
      self.open(f'for (unsigned ei = g; ei < {te}u; ei += {groups}u)')
      self.w(f'const float* bq = cur + {stage_off[t.B.name]} + ei * {bvals}u + l;')
      self.w(f'const float4* rq4 = reinterpret_cast<const float4*>(cur + {stage_off[t.R.name]} + ei * {rvals}u);')
      P = t.P
      for m in range(P):
        self.w(f'const float q{m} = bq[{m * t.K}];')
      nr = t.R.storage_size()
      for v in range((nr + 3) // 4):
        self.w(f'const float4 r{v} = rq4[{v}];')
      comp = ['x', 'y', 'z', 'w']
      look = t.R.sparse_lookup() if t.R.sparse else None
      for j in range(s.N):
        expr = '0.0f'
        for m in range(P):
          pos = (look.get((m, j)) if look is not None else j * P + m)
          if pos is not None:
            expr = f'fmaf(q{m}, r{pos // 4}.{comp[pos % 4]}, {expr})'
        self.w(f'{ubuf}[(ei * {s.N}u + {j}u) * {pitch}u + l] = {expr};')
      self.close()
      self.close()
      self.w(f'tfb_tc::named_sync(1, {NP});')
    # lane phase: wait for the slot, read the lane's column, split, store to TMEM
    if t.R is not None:
      src = f'({ubuf} + row * {pitch}u)'
      vec = True
    else:
      src = f'(cur + {stage_off[t.B.name]} + le * {bvals}u + lj * {t.K}u)'
      vec = t.K % 4 == 0
    self._lane(ti, t, slot_col, lim, src, vec)
    # the transposition buffer of this term is reused two terms later (or next term with one
    # buffer), and the stage / buffers are reused after the last term
    if self.sm['nbuf'] == 1 or ti == len(s.terms) - 1:
      self.w(f'tfb_tc::named_sync(1, {NP});')
    self.close()

  def _ahead_ok(self):
    return (self.prec == 'tf32x3' and self.LC == 16 and
            all(t.K % 4 == 0 and -(-self.lay['kpad'][ti] // 16) <= self.H for ti, t in enumerate(self.s.terms)))

  def _lanes_ahead(self, slot_base, lim):
    """Lane phases of all terms with the next term's column read and split while the
    previous term's tensor-memory stores complete (plan option `ahead`). Two register sets
    alternate; per thread the slot waits, stores and FULL arrivals keep the order of the
    per-term lane phase."""
    b, s = self.base, self.s
    pitch = self.sm['pitch']
    nterms = len(s.terms)
    self.open('')
    self.w('const unsigned c0 = grp * 16u;')
    self.w('unsigned hv0[16], lv0[16], hv1[16], lv1[16];')

    def load_split(ti, reg):
      t = s.terms[ti]
      self.open('')
      self.w('float u[16];')
      self.w('#pragma unroll')
      self.w('for (int i = 0; i < 16; ++i) u[i] = 0.0f;')
      self.open(f'if (active && c0 < {self.lay["kpad"][ti]}u)')
      self.w(f'const float* p = (ubuf{ti} + row * {pitch}u) + c0;')
      for v in range(4):
        self.w(f'if (c0 + {4 * v}u < {t.K}u) {{ const float4 x = *reinterpret_cast<const float4*>(p + {4 * v}); '
               f'u[{4*v}] = x.x; u[{4*v+1}] = x.y; u[{4*v+2}] = x.z; u[{4*v+3}] = x.w; }}')
      self.close()
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < 16; ++i) {{ hv{reg}[i] = tfb_tc::tf32_rna(u[i]); '
             f'lv{reg}[i] = __float_as_uint(u[i] - __uint_as_float(hv{reg}[i])); }}')
      self.close()

    load_split(0, 0)
    for ti in range(nterms):
      reg = ti % 2
      kp = self.lay['kpad'][ti]
      acols = self.lay['a_cols'][ti]
      slot_col = slot_base[ti]
      self.w(f'if (it > 0 && !tfb_tc::{self.wfn}(&bars[{nterms + ti}], (it - 1u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, {30 + ti}u); }}')
      self.w('tfb_tc::fence_after();')
      self.open(f'if (c0 < {kp}u)')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col}u + c0, hv{reg});')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols}u + c0, lv{reg});')
      self.open(f'if (c0 + 8u < {kp}u)')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + 8}u + c0, hv{reg} + 8);')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols + 8}u + c0, lv{reg} + 8);')
      self.close()
      self.close()
      if ti + 1 < nterms:
        load_split(ti + 1, (ti + 1) % 2)
      self.w('tfb_tc::st_wait();')
      self.w('tfb_tc::fence_before();')
      self.w(f'tfb_tc::mbar_arrive(&bars[{ti}]);')
    self.close()

  def _lane(self, ti, t, slot_col, lim, src, vec):
    """Lane phase of term ti: wait for its TMEM slot, read the lane's column of U_t from
    `src`, split it into hi + lo and store both with tcgen05.st, then arrive on FULL[ti]."""
    b, LC, H, prec = self.base, self.LC, self.H, self.prec
    kp = self.lay['kpad'][ti]
    acols = self.lay['a_cols'][ti]
    nterms = len(self.s.terms)
    self.w(f'if (it > 0 && !tfb_tc::{self.wfn}(&bars[{nterms + ti}], (it - 1u) & 1u, {lim}ull)) {{ ok = false; atomicMax(&tfb_err_{b}, {30 + ti}u); }}')
    self.w('tfb_tc::fence_after();')
    if self.pipe == 2 and prec == 'tf32x3' and vec and t.K % 4 == 0 and LC == 16 and -(-kp // LC) <= H:
      # one body for all groups: group g takes columns [16 g, 16 g + 16) of the slot (keeps
      # the instruction footprint of the lane phase to one copy per term)
      self.open('')
      self.w('const unsigned c0 = grp * 16u;')
      self.open(f'if (c0 < {kp}u)')
      self.w('float u[16];')
      self.w('#pragma unroll')
      self.w('for (int i = 0; i < 16; ++i) u[i] = 0.0f;')
      self.open('if (active)')
      self.w(f'const float* p = {src} + c0;')
      for v in range(4):
        self.w(f'if (c0 + {4 * v}u < {t.K}u) {{ const float4 x = *reinterpret_cast<const float4*>(p + {4 * v}); '
               f'u[{4*v}] = x.x; u[{4*v+1}] = x.y; u[{4*v+2}] = x.z; u[{4*v+3}] = x.w; }}')
      self.close()
      self.w('unsigned hv[16], lv[16];')
      self.w('#pragma unroll')
      self.w('for (int i = 0; i < 16; ++i) { hv[i] = tfb_tc::tf32_rna(u[i]); lv[i] = __float_as_uint(u[i] - __uint_as_float(hv[i])); }')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col}u + c0, hv);')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols}u + c0, lv);')
      self.open(f'if (c0 + 8u < {kp}u)')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + 8}u + c0, hv + 8);')
      self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols + 8}u + c0, lv + 8);')
      self.close()
      self.close()
      self.close()
      self.w('tfb_tc::st_wait();')
      self.w('tfb_tc::fence_before();')
      self.w(f'tfb_tc::mbar_arrive(&bars[{ti}]);')
      return
    for ci, l0 in enumerate(range(0, kp, LC)):
      n = min(LC, kp - l0)
      real = max(0, min(n, t.K - l0))
      self.open(f'if (grp == {ci % H}u)')
      self.w(f'float u[{n}];')
      self.w('#pragma unroll')
      self.w(f'for (int i = 0; i < {n}; ++i) u[i] = 0.0f;')
      if real > 0:
        self.open('if (active)')
        self.w(f'const float* p = {src} + {l0};')
        if vec and l0 % 4 == 0:
          for v in range(real // 4):
            self.w(f'{{ const float4 x = *reinterpret_cast<const float4*>(p + {4 * v}); '
                   f'u[{4*v}] = x.x; u[{4*v+1}] = x.y; u[{4*v+2}] = x.z; u[{4*v+3}] = x.w; }}')
          for i in range(real // 4 * 4, real):
            self.w(f'u[{i}] = p[{i}];')
        else:
          self.w('#pragma unroll')
          self.w(f'for (int i = 0; i < {real}; ++i) u[i] = p[i];')
        self.close()
      if prec == 'tf32x3':
        self.w(f'unsigned hv[{n}], lv[{n}];')
        self.w('#pragma unroll')
        self.w(f'for (int i = 0; i < {n}; ++i) {{ hv[i] = tfb_tc::tf32_rna(u[i]); lv[i] = __float_as_uint(u[i] - __uint_as_float(hv[i])); }}')
        for c8 in range(0, n, 8):
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + l0 + c8}u, hv + {c8});')
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols + l0 + c8}u, lv + {c8});')
      else:
        half = n // 2
        self.w(f'unsigned hv[{half}], lv[{half}];')
        self.w('#pragma unroll')
        self.open(f'for (int i = 0; i < {half}; ++i)')
        self.w('const __nv_bfloat16 h0 = __float2bfloat16_rn(u[2 * i]), h1 = __float2bfloat16_rn(u[2 * i + 1]);')
        self.w('const __nv_bfloat16 l0_ = __float2bfloat16_rn(u[2 * i] - __bfloat162float(h0));')
        self.w('const __nv_bfloat16 l1_ = __float2bfloat16_rn(u[2 * i + 1] - __bfloat162float(h1));')
        self.w('hv[i] = (unsigned)__bfloat16_as_ushort(h0) | ((unsigned)__bfloat16_as_ushort(h1) << 16);')
        self.w('lv[i] = (unsigned)__bfloat16_as_ushort(l0_) | ((unsigned)__bfloat16_as_ushort(l1_) << 16);')
        self.close()
        for c8 in range(0, half, 8):
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + l0 // 2 + c8}u, hv + {c8});')
          self.w(f'tfb_tc::st_x8(lane_addr + {slot_col + acols + l0 // 2 + c8}u, lv + {c8});')
      self.close()
    self.w('tfb_tc::st_wait();')
    self.w('tfb_tc::fence_before();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{ti}]);')

  def _epilogue(self, d_main, d_corr, NP, sbuf='ubuf0', final_sync=True):
    """Epilogue of the previous tile: accumulators -> registers (then FREE for the MMA), sum,
    and either stage in `sbuf` + one bulk store (strided, aligned, unmasked output) or
    per-lane stores. With final_sync=False the staging buffer's reuse is left to the caller.
    """
    s = self.s
    M = s.M
    H = self.H
    te = self.sm['te']
    nld = (M + 7) // 8
    per = (nld + H - 1) // H
    out = s.out
    self.w(f'unsigned dv[{per * 8}], dc[{per * 8}];')
    for k in range(per):
      blk = f'8u * (grp + {k * H}u < {nld}u ? grp + {k * H}u : 0u)'
      self.w(f'tfb_tc::ld_x8(lane_addr + {d_main}u + {blk}, dv + {8 * k});')
      self.w(f'tfb_tc::ld_x8(lane_addr + {d_corr}u + {blk}, dc + {8 * k});')
    self.w('tfb_tc::ld_wait();')
    self.w('tfb_tc::fence_before();')
    self.w(f'tfb_tc::mbar_arrive(&bars[{2 * len(s.terms) + 1}]);')
    self.w('#pragma unroll')
    self.w(f'for (int i = 0; i < {per * 8}; ++i) dv[i] = __float_as_uint(__uint_as_float(dv[i]) + __uint_as_float(dc[i]));')
    self.w(f'const size_t pe0 = prev_tile * {te}u;')
    self.w('const size_t pel = pe0 + le;')
    self.w('const bool pvalid = lane_col && pel < numElements;')
    bulk_ok = (out.addressing.name == 'STRIDED' and not s.accumulate
               and out.element_volume() == M * s.N and out.element_volume() % 4 == 0)
    last = M - 8 * (nld - 1)
    if bulk_ok:
      # stage the tile's output contiguously and write it with one bulk copy
      self.w(f'float* const obase = {out.name} + pe0 * {out.element_volume()}u + {out.name}_extraOffset;')
      self.w(f'const size_t nvalid = (numElements - pe0) < {te}u ? (numElements - pe0) : {te}u;')
      self.w('const bool bulk = flags == nullptr && ((reinterpret_cast<uintptr_t>(obase) & 15u) == 0u);')
      self.open('if (bulk)')
      self.open('if (pvalid)')
      for k in range(per):
        self.w(f'const unsigned q{k} = grp + {k * H}u;')
        self.open(f'if (q{k} < {nld}u)')
        self.w(f'float* const dst = {sbuf} + row * {M}u + 8u * q{k};')
        if M % 8 == 0:
          self.w(f'reinterpret_cast<float4*>(dst)[0] = make_float4(__uint_as_float(dv[{8*k}]), __uint_as_float(dv[{8*k+1}]), __uint_as_float(dv[{8*k+2}]), __uint_as_float(dv[{8*k+3}]));')
          self.w(f'reinterpret_cast<float4*>(dst)[1] = make_float4(__uint_as_float(dv[{8*k+4}]), __uint_as_float(dv[{8*k+5}]), __uint_as_float(dv[{8*k+6}]), __uint_as_float(dv[{8*k+7}]));')
        else:
          self.w(f'const unsigned cnt = (q{k} == {nld - 1}u) ? {last}u : 8u;')
          self.w(f'for (unsigned i = 0; i < cnt; ++i) dst[i] = __uint_as_float(dv[{8 * k} + i]);')
        self.close()
      self.close()
      self.w('tfb_tc::fence_proxy_async();')
      self.w(f'tfb_tc::named_sync(1, {NP});')
      self.open('if (ptid == 0)')
      self.w(f'tfb_tc::bulk_store(obase, {sbuf}, (unsigned)(nvalid * {out.element_volume() * 4}u));')
      self.w('tfb_tc::bulk_wait_read();')
      self.close()
      if final_sync:
        self.w(f'tfb_tc::named_sync(1, {NP});')
      self.close()
      self.open('else if (pvalid && (flags == nullptr || flags[pel] != 0u))')
    else:
      self.open('if (pvalid && (flags == nullptr || flags[pel] != 0u))')
    self.w(f'float* const col = {self._elem_ptr(out, "pel")} + (size_t)lj * {M}u;')
    for k in range(per):
      self.w(f'const unsigned q{k} = grp + {k * H}u;')
      self.open(f'if (q{k} < {nld}u)')
      self.w(f'float* const dst = col + 8u * q{k};')
      self.w(f'const unsigned cnt = (q{k} == {nld - 1}u) ? {last}u : 8u;')
      if s.accumulate:
        self.w(f'for (unsigned i = 0; i < cnt; ++i) dst[i] += __uint_as_float(dv[{8 * k} + i]);')
      else:
        self.w(f'for (unsigned i = 0; i < cnt; ++i) dst[i] = __uint_as_float(dv[{8 * k} + i]);')
      self.close()
    self.close()
