"""Throughput of the fused signature-kernel Gram on B200.

Workload (one step): the normalised truncated signature Gram K(X, Y) of
N = M = 512 sequences per GPU, L = 200 points, d = 8 random-walk channels
(cumsum of N(0, 1/L) increments) plus a linear time channel, RBF static
kernel with bandwidth sqrt(8), n_levels = 5, order = 1, normalize = True,
FP32 inputs (FP32 kernels with FP64 level sums and normalisation).  A step
computes the 512 x 512 Gram plus the two 512-entry diagonal passes that
normalisation needs, i.e. the whole ``SignatureKernel(...)(X, Y)`` call.

Metric: Gram entries per second (N*M per step, summed over ranks).  With
``--gpus N`` under torchrun every rank computes its own 512 x 512 block
(weak scaling, no data-path collective).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

``--impl reference`` times the reference recursion on the host cores (the
NumPy restatement in ``oracle/`` run over a process pool, since the
reference itself needs CuPy on a GPU) on the same workload, one bounded
sample of pairs per step.
"""

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

N_SEQ = 512       # sequences per side (--n-seq shrinks it for profiling only)
SEQ_LEN = 200
D_WALK = 8
N_LEVELS = 5
ORDER = 1
BANDWIDTH = math.sqrt(8.0)
METRIC = 'Gram entries/sec & fwd+bwd s/step, mixed vs plain FP32 on B200 @1e-5 vs FP64'
UNIT = 'Gram entries/s'
WORKLOAD = 'sig_dp_rbf_N512_M512_L200_d9_m5_p1_normalized'


def make_walks(n, L, d, seed):
  """Random walks (cumsum of N(0, 1/L) increments) + a time channel."""
  rng = np.random.default_rng(seed)
  inc = rng.standard_normal((n, L - 1, d)) / np.sqrt(L)
  X = np.concatenate([np.zeros((n, 1, d)), np.cumsum(inc, 1)], 1)
  t = np.broadcast_to(np.linspace(0, 1, L)[None, :, None], (n, L, 1))
  return np.concatenate([X, t], -1).astype(np.float32)


def config(n_gpus, extra=None):
  c = {'workload': WORKLOAD, 'n_x': N_SEQ, 'n_y': N_SEQ, 'seq_len': SEQ_LEN,
       'd': D_WALK + 1, 'n_levels': N_LEVELS, 'order': ORDER,
       'static_kernel': 'rbf', 'bandwidth': BANDWIDTH, 'normalize': True,
       'global_pairs': N_SEQ * N_SEQ * n_gpus,
       'parallelism': f'pairs-sharded x{n_gpus}' if n_gpus > 1 else 'single'}
  if extra:
    c.update(extra)
  return c


# ---------------------------------------------------------------------------
# Host CPU baseline: the reference recursion restated in NumPy (oracle/).
# ---------------------------------------------------------------------------

def _cpu_chunk(args):
  X, Y = args
  sys.path.insert(0, ROOT)
  from oracle import ksig_oracle as O
  return O.signature_kernel(X, Y, n_levels=N_LEVELS, order=ORDER,
                            normalize=True, param=BANDWIDTH)


def cpu_sample(nx, ny, seed, pool=None):
  """Times the oracle on an nx x ny block (plus its diagonal passes)."""
  X = make_walks(nx, SEQ_LEN, D_WALK, seed).astype(np.float64)
  Y = make_walks(ny, SEQ_LEN, D_WALK, seed + 1).astype(np.float64)
  t0 = time.perf_counter()
  if pool is None:
    _cpu_chunk((X, Y))
  else:
    rows = np.array_split(np.arange(nx), len(pool._pool))
    list(pool.map(_cpu_chunk, [(X[r], Y) for r in rows if len(r)]))
  return time.perf_counter() - t0


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------

class ClockSampler:
  FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
            'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
            'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

  def __init__(self, gpu_index):
    self.idx = gpu_index
    self.proc = None
    self.path = None

  def start(self):
    try:
      # Raw samples go to KSIG_CLOCKS_DIR (default: the system temp dir);
      # the JSON line carries their summary.
      out_dir = os.environ.get('KSIG_CLOCKS_DIR') or tempfile.gettempdir()
      os.makedirs(out_dir, exist_ok=True)
      self.path = os.path.join(out_dir, f'clocks_gpu{self.idx}.csv')
      self.f = open(self.path, 'w')
      self.proc = subprocess.Popen(
          ['nvidia-smi', f'--id={self.idx}', f'--query-gpu={self.FIELDS}',
           '--format=csv,noheader,nounits', '-lms', '100'],
          stdout=self.f, stderr=subprocess.DEVNULL)
    except Exception:  # noqa: BLE001 - clocks are best effort
      self.proc = None

  def stop(self):
    if self.proc is None:
      return None
    self.proc.terminate()
    try:
      self.proc.wait(timeout=5)
    except Exception:  # noqa: BLE001
      self.proc.kill()
    self.f.close()
    sm, mx, reasons = [], None, set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
             'sw_power_cap']
    with open(self.path) as f:
      for line in f:
        parts = [p.strip() for p in line.split(',')]
        if len(parts) < 9:
          continue
        try:
          sm.append(float(parts[1]))
          mx = float(parts[2])
        except ValueError:
          continue
        for n, v in zip(names, parts[5:9]):
          if v.lower() == 'active':
            reasons.add(n)
    if not sm:
      return None
    return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': mx,
            'reasons': sorted(reasons), 'samples': len(sm)}


# ---------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------

def _other_bounds(traffic, k_ms):
  """HBM and tensor-core fractions of the sweep against MEASURED_PEAKS.json
  (driver-measured copy bandwidth and bf16 GEMM rate of this pool)."""
  path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
  src = 'MEASURED_PEAKS.json'
  try:
    with open(path) as f:
      pk = json.load(f)
  except (OSError, ValueError):
    # Without the measured file: an earlier B200 measurement (STREAM-style
    # copy 6.65 TB/s, cuBLAS bf16 burst 1.59 PFLOP/s), reported as fallback.
    pk = {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0}
    src = 'fallback (no MEASURED_PEAKS.json): 6.65 TB/s copy, 1.59 PFLOP/s bf16'
  out = {'tensor': {'achieved': 0.0, 'peak': pk.get('bf16_tflops'), 'unit': 'TFLOP/s',
                    'frac': 0.0, 'note': 'no tensor-core work (d <= 16 dot products)',
                    'source': src}}
  if traffic and k_ms:
    gbs = traffic / (k_ms * 1e-3) / 1e9
    out['hbm'] = {'achieved': gbs, 'peak': pk.get('hbm_gbs'), 'unit': 'GB/s',
                  'frac': gbs / pk['hbm_gbs'] if pk.get('hbm_gbs') else None,
                  'source': src}
  return out


def bwd_roofline(bwd_ms, peak):
  """Roofline of the one-launch DP adjoint on the 512 x 512 levels.

  Algorithmic flops per pair, with G = L^2 grid points and cells = (L-1)^2:
    phase 1 (forward recomputed):  G (2d + 4) + cells (4 + 4 (m - 1))
    phase 2 Gram recomputed:       G (2d + 4)
    state recovery by subtraction: cells 2 (m - 1)
    adjoint recursion:             cells (5 (m - 1) + 2)
    pull-back to dX:               G (2d + 6)
  The per-step records (phase 1 writes, phase 2 reads (L + 33) (m - 1)
  FP32 values per lane and strip) are the adjoint's own intermediate, not
  input bytes."""
  d = D_WALK + 1
  m = N_LEVELS
  G = SEQ_LEN * SEQ_LEN
  cells = (SEQ_LEN - 1) ** 2
  flops = (2 * G * (2 * d + 4) + G * (2 * d + 6)
           + cells * ((4 + 4 * (m - 1)) + 2 * (m - 1) + 5 * (m - 1) + 2))
  achieved = flops * N_SEQ * N_SEQ / (bwd_ms * 1e-3) / 1e12
  rec = (SEQ_LEN + 33) * (m - 1) * 32 * 4
  traffic = None
  tpath = os.path.join(ROOT, 'profiles', 'dp_bwd_traffic.json')
  if os.path.exists(tpath):
    with open(tpath) as f:
      traffic = json.load(f).get('bytes_per_launch')
  return {'bound': 'fp32', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
          'frac': achieved / peak if peak else None,
          'kernel': 'dp_bwd_kernel (one launch, both phases, 512x512 pairs)',
          'kernel_ms': bwd_ms, 'flops_per_pair': flops,
          'record_bytes_per_pair': 2 * rec,
          'traffic': traffic,
          'traffic_source': ('ncu capture committed as profiles/dp_bwd_traffic.json '
                             '(not measured in this run)') if traffic else None}


def run_ours(args, rank, world, dist):
  import torch

  import ksig_b200 as K
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as Lb

  dev = torch.device('cuda', torch.cuda.current_device())
  X = make_walks(N_SEQ, SEQ_LEN, D_WALK, 2 + 2 * rank)
  Y = make_walks(N_SEQ, SEQ_LEN, D_WALK, 3 + 2 * rank)
  Xd = torch.as_tensor(X, device=dev)
  Yd = torch.as_tensor(Y, device=dev)
  kern = K.SignatureKernel(n_levels=N_LEVELS, order=ORDER, normalize=True,
                           static_kernel=K.RBFKernel(BANDWIDTH))
  lib = Lb.lib()
  flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

  def step():
    return kern(Xd, Yd, return_on_gpu=True)

  def barrier():
    if dist is not None:
      dist.barrier()
    torch.cuda.synchronize()

  for _ in range(args.warmup):
    step()
  barrier()
  stream = torch.cuda.current_stream()
  evs = [(torch.cuda.Event(enable_timing=True),
          torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
  clocks = ClockSampler(dev.index if dev.index is not None else 0)
  clocks.start()
  launches0 = lib.ksig_launch_count()
  barrier()
  for i in range(args.steps):
    flush.fill_(i & 0xff)  # evict L2 (126 MB) between steps, untimed
    evs[i][0].record(stream)
    step()
    evs[i][1].record(stream)
  barrier()
  launches = lib.ksig_launch_count() - launches0
  clk = clocks.stop()
  ms = [a.elapsed_time(b) for a, b in evs]
  t_step = sum(ms) / len(ms)
  if dist is not None:
    t = torch.tensor([t_step], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_step = float(t.item())

  # Dominant kernel: the 512 x 512 pair sweep, timed alone with CUDA events
  # recorded by the library on its launch stream.
  Xs, Ys = E.Seqs(Xd), E.Seqs(Yd)
  lib.ksig_profile_read(None, None)
  lib.ksig_profile_enable(1)
  nrep = 5
  for _ in range(nrep):
    flush.fill_(1)
    E.sig_levels(Xs, Ys, Lb.PAIRS_FULL, N_LEVELS, ORDER, True, Lb.STATIC_RBF,
                 BANDWIDTH)
  torch.cuda.synchronize()
  lib.ksig_profile_enable(0)
  tot = ctypes.c_double(0)
  cnt = ctypes.c_longlong(0)
  lib.ksig_profile_read(ctypes.byref(tot), ctypes.byref(cnt))
  k_ms = tot.value / max(cnt.value, 1)
  peak = ctypes.c_double(0)
  Lb.check(lib.ksig_fp32_peak(ctypes.byref(peak),
                              ctypes.c_void_p(stream.cuda_stream)))
  d = D_WALK + 1
  G = SEQ_LEN * SEQ_LEN
  cells = (SEQ_LEN - 1) ** 2
  flops_pair = G * (2 * d + 4) + cells * (4 + 4 * (N_LEVELS - 1))
  achieved = flops_pair * N_SEQ * N_SEQ / (k_ms * 1e-3) / 1e12
  traffic = None
  tpath = os.path.join(ROOT, 'profiles', 'dp_fwd_traffic.json')
  if os.path.exists(tpath):
    with open(tpath) as f:
      traffic = json.load(f).get('bytes_per_launch')

  # The plain FP32 one-pair-per-block baseline kernel on the same 512 x 512
  # level computation (the 'plain' side of 'mixed vs plain FP32').
  plain_ms = None
  if not args.no_plain:
    E.sig_levels_plain(Xs, Ys, Lb.PAIRS_FULL, N_LEVELS, ORDER, Lb.STATIC_RBF,
                       BANDWIDTH)
    torch.cuda.synchronize()
    pm = []
    for _ in range(2):
      flush.fill_(2)
      a = torch.cuda.Event(enable_timing=True)
      b = torch.cuda.Event(enable_timing=True)
      a.record(stream)
      E.sig_levels_plain(Xs, Ys, Lb.PAIRS_FULL, N_LEVELS, ORDER,
                         Lb.STATIC_RBF, BANDWIDTH)
      b.record(stream)
      b.synchronize()
      pm.append(a.elapsed_time(b))
    plain_ms = sum(pm) / len(pm)

  # The adjoints on the same 512 x 512 levels: fused (skewed two-phase sweep)
  # and plain one-pair-per-block, each on random level weights.
  bwd_ms = plain_bwd_ms = None
  if not args.no_plain and not args.no_bwd:
    gl = torch.randn((N_LEVELS + 1, N_SEQ * N_SEQ), device=dev, dtype=torch.float64)

    def timed_once(fn, reps):
      out = []
      for _ in range(reps):
        flush.fill_(3)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        out.append(a.elapsed_time(b))
      return sum(out) / len(out)

    fb = lambda: E.sig_levels_bwd(Xs, Ys, Lb.PAIRS_FULL, N_LEVELS, ORDER,  # noqa: E731
                                  Lb.STATIC_RBF, BANDWIDTH, gl, want_dparam=False)
    fb()
    bwd_ms = timed_once(fb, 3)
    pb = lambda: E.sig_levels_bwd_plain(Xs, Ys, Lb.PAIRS_FULL, N_LEVELS, ORDER,  # noqa: E731
                                        Lb.STATIC_RBF, BANDWIDTH, gl, want_dparam=False)
    plain_bwd_ms = timed_once(pb, 1)

  # End to end through the public API from pinned host memory.
  Xh = torch.as_tensor(X).pin_memory()
  Yh = torch.as_tensor(Y).pin_memory()
  for _ in range(2):
    kern(Xh, Yh)
  barrier()
  e_ms = []
  for i in range(args.steps):
    flush.fill_(i & 0xff)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    Kh = kern(Xh, Yh)  # H2D of X, Y; D2H of the [512, 512] result
    b.record(stream)
    b.synchronize()
    e_ms.append(a.elapsed_time(b))
  e_step = sum(e_ms) / len(e_ms)
  if dist is not None:
    t = torch.tensor([e_step], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e_step = float(t.item())
  assert Kh.shape == (N_SEQ, N_SEQ)

  # Forward + backward (gradient of sum(W * K) w.r.t. X through the adjoint
  # kernels), the 'fwd+bwd s/step' half of the metric.
  fb_ms = None
  fb_steps_ms = None
  split_used = None
  if not args.no_bwd:
    Xg = Xd.clone().requires_grad_(True)
    Wt = torch.randn((N_SEQ, N_SEQ), device=dev, dtype=torch.float32)

    def fb_step():
      Xg.grad = None
      Kg = kern(Xg, Yd, return_on_gpu=True)
      (Kg * Wt).sum().backward()
      return Xg.grad

    for _ in range(3):
      fb_step()
    barrier()
    rec0 = dict(E.REC_STATS)
    fbs = []
    for i in range(args.bwd_steps):
      flush.fill_(i & 0xff)
      a = torch.cuda.Event(enable_timing=True)
      b = torch.cuda.Event(enable_timing=True)
      a.record(stream)
      fb_step()
      b.record(stream)
      b.synchronize()
      fbs.append(a.elapsed_time(b))
    fb_ms = sum(fbs) / len(fbs)
    fb_steps_ms = [round(v, 3) for v in fbs]
    # Timed steps whose forward kept the split gradient pass's records (the
    # backward replays them) and those that ran the one-launch adjoint.
    split_used = {k: E.REC_STATS[k] - rec0[k] for k in rec0}
    if dist is not None:
      t = torch.tensor([fb_ms], device=dev, dtype=torch.float64)
      dist.all_reduce(t, op=dist.ReduceOp.MAX)
      fb_ms = float(t.item())

  cpu = None
  if rank == 0 and world == 1 and not args.no_cpu:
    n = args.cpu_pairs
    secs = cpu_sample(n, n, 100)
    cpu = {'value': n * n / secs, 'unit': UNIT, 'cores': 1, 'kind': 'port',
           'sample': f'{n}x{n} pairs of the same workload (+ diagonal passes),'
                     ' NumPy FP64 restatement of the reference recursion '
                     '(oracle/ksig_oracle.py), single process',
           'seconds': secs}

  # The large ragged order-2 workload (one GPU): forward and forward +
  # input gradient, fused vs plain on a sample, errors against the oracle.
  ragged = None
  if world == 1 and not args.no_ragged:
    ragged = ragged_record(args)

  entries = N_SEQ * N_SEQ * world
  if rank == 0:
    line = {
        'metric': METRIC, 'value': entries / (t_step * 1e-3), 'unit': UNIT,
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': t_step, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': config(world),
        'l2': 'flushed (256 MB write) between timed steps',
        'roofline': {'bound': 'fp32', 'achieved': achieved,
                     'peak': peak.value, 'unit': 'TFLOP/s',
                     'frac': achieved / peak.value if peak.value else None,
                     'traffic': traffic,
                     'traffic_source': 'dram__bytes_read.sum + dram__bytes_write.sum of '
                                       'one ncu capture of this launch, committed as '
                                       'profiles/dp_fwd_traffic.json (not measured in '
                                       'this run)' if traffic else None,
                     'kernel': 'dp_fwd_kernel (512x512 pair sweep)',
                     'kernel_ms': k_ms,
                     'peak_source': 'measured live: FP32 FMA-chain probe '
                                    '(ksig_fp32_peak) on this GPU',
                     # The other two ceilings, for context: the kernel moves
                     # ~10 MB of DRAM per launch and issues no tensor work.
                     'other_bounds': _other_bounds(traffic, k_ms)},
        'e2e': {'value': entries / (e_step * 1e-3), 'unit': UNIT,
                'ms_per_step': e_step,
                'h2d_bytes_per_step': int(X.nbytes + Y.nbytes),
                'd2h_bytes_per_step': int(N_SEQ * N_SEQ * 4)},
        'plain_fp32': None if plain_ms is None else {
            'kernel_ms': plain_ms, 'fused_kernel_ms': k_ms,
            'speedup': plain_ms / k_ms,
            'bwd_kernel_ms': plain_bwd_ms, 'fused_bwd_kernel_ms': bwd_ms,
            'speedup_bwd': (plain_bwd_ms / bwd_ms) if bwd_ms else None,
            'speedup_fwd_bwd': ((plain_ms + plain_bwd_ms) / (k_ms + bwd_ms))
                               if bwd_ms else None,
            'what': 'plain FP32 one-pair-per-block kernels '
                    '(ksig_signature_kern_plain, ksig_signature_kern_plain_bwd) '
                    'against the fused sweep and adjoint on the same 512x512 levels'},
        'roofline_bwd': None if bwd_ms is None else bwd_roofline(bwd_ms, peak.value),
        'fwd_bwd': None if fb_ms is None else {
            's_per_step': fb_ms * 1e-3, 'ms_per_step': fb_ms,
            'what': 'K(X, Y) forward + dL/dX backward (L = sum W*K), '
                    'X [512, 200, 9] requires grad', 'steps': args.bwd_steps,
            'step_ms': fb_steps_ms,
            'median_ms': statistics.median(fb_steps_ms) if fb_steps_ms else None,
            'split_pass': split_used},
        'gpu_launches': int(launches),
        'clocks': clk,
        'cpu_baseline': cpu,
        'ragged_dp': ragged,
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Ragged higher-order workload (not the default bench line): N = M = 2048
# sequences, lengths log-uniform in [32, 1024], d = 16 cumsummed N(0, 1)
# increments, RBF bandwidth sqrt(16), n_levels = 8, order = 2, normalize.
# Times the forward Gram and forward + input gradient through the public API
# (ragged lists), and the fused and plain kernels on a bounded sample of the
# same pairs.
# ---------------------------------------------------------------------------

RAGGED = dict(n=2048, lmin=32, lmax=1024, d=16, n_levels=8, order=2, bw=4.0)


def make_ragged(n, lmin, lmax, d, seed):
  rng = np.random.default_rng(seed)
  lens = np.exp(rng.uniform(np.log(lmin), np.log(lmax), n)).astype(np.int64)
  lens = np.clip(lens, lmin, lmax)
  return [np.cumsum(rng.standard_normal((int(L), d)), 0).astype(np.float32)
          for L in lens]


def _sample_errors(kern, R, Xl, Yl, dev):
  """Per-entry errors on the sample whose FP64 oracle values are committed
  in tests/golden/ragged_dp_sample.npz (written by make_ragged_sample.py
  from the same seeded batch): the normalised K of 4 x 4 pairs holding the
  longest sequences of each side, and dL/dX of 2 x 2 of them."""
  import torch
  path = os.path.join(ROOT, 'tests', 'golden', 'ragged_dp_sample.npz')
  if not os.path.exists(path):
    return None
  f = np.load(path)
  Xs = [Xl[i] for i in f['ix']]
  Ys = [Yl[i] for i in f['iy']]
  K = kern(Xs, Ys, return_on_gpu=True).double().cpu().numpy()
  ref = f['K']
  k_err = float(np.max(np.abs(K - ref) / np.abs(ref)))
  Xg = [Xl[i].clone().requires_grad_(True) for i in f['gx']]
  Yg = [Yl[i] for i in f['gy']]
  W = torch.tensor(f['W'], device=dev, dtype=torch.float32)
  (kern(Xg, Yg, return_on_gpu=True) * W).sum().backward()
  g_err = 0.0
  for j, x in enumerate(Xg):
    g = x.grad.double().cpu().numpy()
    r = f['dX'][j, :g.shape[0]]
    floor = 1e-2 * np.max(np.abs(r))
    g_err = max(g_err, float(np.max(np.abs(g - r) / np.maximum(np.abs(r), floor))))
  return {'pairs': int(len(Xs) * len(Ys)),
          'lengths_x': [int(Xl[i].shape[0]) for i in f['ix']],
          'lengths_y': [int(Yl[i].shape[0]) for i in f['iy']],
          'max_rel_err_K': k_err,
          'max_rel_err_dX': g_err,
          'dX_pairs': int(len(Xg) * len(Yg)),
          'bar': 'K: |err| / |ref| per entry (target 1e-5); dX: |err| / '
                 'max(|ref|, 1e-2 max|ref|) per coordinate (target 1e-4)',
          'reference': 'FP64 oracle (oracle/ksig_oracle.py, autograd through '
                       'oracle/ksig_oracle_torch.py) on the FP32-rounded inputs, '
                       'committed as tests/golden/ragged_dp_sample.npz'}


def ragged_record(args, fwd_steps=1, bwd_steps=1):
  """Times the ragged order-2 workload through the public API (lists of
  device tensors): forward, and forward + input gradient; the fused and plain
  kernels on a bounded sample of the same pairs; and the per-entry errors of
  the oracle sample."""
  import torch

  import ksig_b200 as K
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as Lb
  R = dict(RAGGED)
  if args.n_seq is not None and args.workload == 'ragged-dp':
    R['n'] = args.n_seq
  n, m, p, bw = R['n'], R['n_levels'], R['order'], R['bw']
  dev = torch.device('cuda', torch.cuda.current_device())
  Xl = [torch.as_tensor(a, device=dev) for a in make_ragged(n, R['lmin'], R['lmax'], R['d'], 5)]
  Yl = [torch.as_tensor(a, device=dev) for a in make_ragged(n, R['lmin'], R['lmax'], R['d'], 6)]
  lx = np.array([a.shape[0] for a in Xl])
  ly = np.array([a.shape[0] for a in Yl])
  cells = float(np.sum(lx - 1)) * float(np.sum(ly - 1))
  kern = K.SignatureKernel(n_levels=m, order=p, normalize=True,
                           static_kernel=K.RBFKernel(bw))
  W = torch.randn((n, n), device=dev, dtype=torch.float32)

  def timed(fn, steps, warm):
    for _ in range(warm):
      fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
      a = torch.cuda.Event(enable_timing=True)
      b = torch.cuda.Event(enable_timing=True)
      a.record()
      fn()
      b.record()
      b.synchronize()
      ts.append(a.elapsed_time(b))
    return sum(ts) / len(ts)

  fwd_ms = timed(lambda: kern(Xl, Yl, return_on_gpu=True), fwd_steps, 1)
  Xg = [a.clone().requires_grad_(True) for a in Xl]

  def fb():
    Kg = kern(Xg, Yl, return_on_gpu=True)
    (Kg * W).sum().backward()

  fb_ms = timed(fb, bwd_steps, 0)

  # Fused vs plain kernels on the same bounded sample of pairs.
  s = min(args.plain_sample, n)
  def seqs(lst):
    L = max(a.shape[0] for a in lst)
    data = torch.zeros((len(lst), L, R['d']), device=dev)
    for i, a in enumerate(lst):
      data[i, :a.shape[0]] = a
    return E.Seqs(data, torch.tensor([a.shape[0] for a in lst], device=dev))
  Xs, Ys = seqs(Xl[:s]), seqs(Yl[:s])
  scells = float(np.sum(lx[:s] - 1)) * float(np.sum(ly[:s] - 1))
  gl = torch.randn((m + 1, s * s), device=dev, dtype=torch.float64)
  os.environ.setdefault('KSIG_PLAIN_SCRATCH_MB', '65536')
  f_fwd = timed(lambda: E.sig_levels(Xs, Ys, Lb.PAIRS_FULL, m, p, True, Lb.STATIC_RBF, bw), 2, 1)
  f_bwd = timed(lambda: E.sig_levels_bwd(Xs, Ys, Lb.PAIRS_FULL, m, p, Lb.STATIC_RBF, bw, gl,
                                         want_dparam=False), 2, 1)
  p_fwd = timed(lambda: E.sig_levels_plain(Xs, Ys, Lb.PAIRS_FULL, m, p, Lb.STATIC_RBF, bw), 1, 0)
  p_bwd = timed(lambda: E.sig_levels_bwd_plain(Xs, Ys, Lb.PAIRS_FULL, m, p, Lb.STATIC_RBF, bw,
                                               gl, want_dparam=False), 1, 0)
  errs = _sample_errors(kern, R, Xl, Yl, dev) if n == RAGGED['n'] else None
  return {
      'workload': f'sig_dp_rbf_ragged_N{n}_M{n}_L32-1024_d16_m{m}_p{p}_normalized',
      'forward': {'value': n * n / (fwd_ms * 1e-3), 'unit': UNIT, 's_per_step': fwd_ms * 1e-3,
                  'cells_per_s': cells / (fwd_ms * 1e-3), 'steps': fwd_steps},
      'fwd_bwd': {'s_per_step': fb_ms * 1e-3, 'steps': bwd_steps,
                  'what': 'K(X, Y) + d sum(W*K)/dX through the public API (ragged lists '
                          'of device tensors)'},
      'plain_vs_fused_sample': {
          'pairs': s * s, 'cells': scells,
          'what': f'the first {s} x {s} pairs: plain FP32 one-pair-per-block kernels '
                  '(ksig_signature_kern_plain / _plain_bwd) against the fused '
                  'forward and adjoint kernels on the same levels',
          'fused_fwd_ms': f_fwd, 'fused_bwd_ms': f_bwd,
          'plain_fwd_ms': p_fwd, 'plain_bwd_ms': p_bwd,
          'speedup_fwd': p_fwd / f_fwd, 'speedup_bwd': p_bwd / f_bwd,
          'speedup_fwd_bwd': (p_fwd + p_bwd) / (f_fwd + f_bwd),
          'plain_fwd_bwd_full_s_est': (p_fwd + p_bwd) * 1e-3 * cells / scells,
          'speedup_fwd_bwd_full_est': (p_fwd + p_bwd) * 1e-3 * cells / scells / (fb_ms * 1e-3)},
      'oracle_sample': errs,
      'cells': cells, 'dtype': 'f32', 'data': 'synthetic (seeded, bench.make_ragged)',
  }


def run_ragged(args):
  line = {'metric': METRIC}
  line.update(ragged_record(args, args.steps, args.bwd_steps))
  print(json.dumps(line))


# Gram forms (not the default bench line): the same DP level computation
# (N = M = 256 random walks + time, L = 200, RBF bandwidth sqrt(d),
# n_levels = 5, order 1) at d = 8, 15, 31 and 63 channels plus time, with
# the static Gram formed three ways:
#   register: fused in the sweep on the FP32 pipe (FFMA2, lane-centred);
#   tensor:   tcgen05 3xTF32 tiles into per-task Gram slots, then the
#             Gram-input sweep (KSIG_FORCE_GIN=1, KSIG_GRAM_TC=1);
#   cuda:     CUDA-core difference tiles into the slots, then the same sweep.
# Reports kernel time per form and the largest level difference against the
# FP64 register path (the forms' oracle errors are in the tests).

def run_gram_forms(args):
  import torch

  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as Lb
  n = args.n_seq or 256
  dev = torch.device('cuda', 0)
  out = {'metric': METRIC, 'workload': f'gram_forms_N{n}_L200_m5_p1', 'forms': {}}

  def timed(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
      a = torch.cuda.Event(enable_timing=True)
      b = torch.cuda.Event(enable_timing=True)
      a.record()
      fn()
      b.record()
      b.synchronize()
      ts.append(a.elapsed_time(b))
    return min(ts)

  dws = [int(v) - 1 for v in args.gram_d.split(',')] if args.gram_d else (8, 15, 31, 63)
  forms = args.gram_forms.split(',') if args.gram_forms else ('register', 'tensor', 'cuda')
  for dw in dws:
    d = dw + 1
    bw = math.sqrt(dw)
    X = torch.as_tensor(make_walks(n, SEQ_LEN, dw, 11), device=dev)
    Y = torch.as_tensor(make_walks(n, SEQ_LEN, dw, 12), device=dev)
    Xs, Ys = E.Seqs(X), E.Seqs(Y)
    ref = E.sig_levels(E.Seqs(X.double()), E.Seqs(Y.double()), Lb.PAIRS_FULL, 5, 1, True,
                       Lb.STATIC_RBF, bw)
    scale = ref.abs().amax(dim=1, keepdim=True).clamp_min(1e-300)
    row = {}
    for form, env in (('register', {}), ('tensor', {'KSIG_FORCE_GIN': '1', 'KSIG_GRAM_TC': '1'}),
                      ('cuda', {'KSIG_FORCE_GIN': '1', 'KSIG_GRAM_TC': '0'})):
      if form not in forms:
        continue
      if form == 'register' and d > 32:
        row[form] = {'unavailable': 'no register-Gram tile above 32 coordinates'}
        continue
      old = {k: os.environ.get(k) for k in ('KSIG_FORCE_GIN', 'KSIG_GRAM_TC')}
      os.environ.update(env)
      try:
        fn = lambda: E.sig_levels(Xs, Ys, Lb.PAIRS_FULL, 5, 1, True, Lb.STATIC_RBF, bw)  # noqa: E731
        lev = fn()
        ms = timed(fn)
        row[form] = {'ms': ms, 'max_level_diff_vs_fp64': float(((lev - ref).abs() / scale).max())}
      except Exception as e:  # noqa: BLE001 - a form without a compiled tile
        row[form] = {'unavailable': str(e)[:120]}
      finally:
        for k, v in old.items():
          if v is None:
            os.environ.pop(k, None)
          else:
            os.environ[k] = v
    out['forms'][f'd={d}'] = row
  print(json.dumps(out))


# Ragged PDE workload (not the default bench line): N = M = 256 Brownian
# paths (N(0, 1/L) increments, d = 3 plus a time channel), lengths uniform
# in [64, 512], dyadic_order = 1, RBF bandwidth 1, normalize.  One call
# through the public API, then the same call captured in a CUDA graph, then
# replayed after the tile-width autotuner.

def make_brownian(n, lmin, lmax, d, seed):
  rng = np.random.default_rng(seed)
  lens = rng.integers(lmin, lmax + 1, n)
  data = np.zeros((n, lmax, d + 1), dtype=np.float32)
  for i, L in enumerate(lens):
    inc = rng.standard_normal((L - 1, d)) / np.sqrt(L)
    data[i, 1:L, :d] = np.cumsum(inc, 0)
    data[i, :L, d] = np.linspace(0, 1, L)
  return data, lens


def run_ragged_pde(args):
  import torch

  import ksig_b200 as K
  from ksig_b200 import tuning
  n = args.n_seq or 256
  dev = torch.device('cuda', 0)
  xd, lx = make_brownian(n, 64, 512, 3, 3)
  yd, ly = make_brownian(n, 64, 512, 3, 4)
  X = K.Ragged(torch.as_tensor(xd, device=dev), torch.as_tensor(lx, device=dev))
  Y = K.Ragged(torch.as_tensor(yd, device=dev), torch.as_tensor(ly, device=dev))
  kern = K.SignaturePDEKernel(dyadic_order=1, static_kernel=K.RBFKernel(1.0))
  F = 2
  cells = float(np.sum(lx - 1)) * float(np.sum(ly - 1)) * F * F

  def timed(fn, steps, warm):
    for _ in range(warm):
      fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
      a = torch.cuda.Event(enable_timing=True)
      b = torch.cuda.Event(enable_timing=True)
      a.record()
      fn()
      b.record()
      b.synchronize()
      ts.append(a.elapsed_time(b))
    return sum(ts) / len(ts)

  eager = timed(lambda: kern(X, Y, return_on_gpu=True), args.steps, args.warmup)
  g = K.GraphedKernel(kern, X, Y)
  graph = timed(g, args.steps, args.warmup)
  tuned = tuning.autotune(kern, X, Y, reps=2)
  gt = K.GraphedKernel(kern, X, Y)
  graph_tuned = timed(gt, args.steps, args.warmup)
  ref = kern(X, Y, return_on_gpu=True)
  tuning.reset()
  # FP32 against the FP64 path on a 16 x 16 corner.
  c = min(16, n)
  X64 = K.Ragged(X.data[:c].double(), X.lengths[:c])
  Y64 = K.Ragged(Y.data[:c].double(), Y.lengths[:c])
  k64 = kern(X64, Y64, return_on_gpu=True)
  k32 = kern(K.Ragged(X.data[:c], X.lengths[:c]), K.Ragged(Y.data[:c], Y.lengths[:c]),
             return_on_gpu=True)
  rel = float(((k32.double() - k64).abs() / k64.abs().clamp_min(1e-300)).max())
  line = {
      'metric': METRIC, 'workload': f'sig_pde_rbf_ragged_N{n}_M{n}_L64-512_d4_dyadic1_normalized',
      'unit': UNIT,
      'eager': {'value': n * n / (eager * 1e-3), 'ms_per_step': eager},
      'graph': {'value': n * n / (graph * 1e-3), 'ms_per_step': graph},
      'graph_autotuned': {'value': n * n / (graph_tuned * 1e-3), 'ms_per_step': graph_tuned,
                          'widths': {str(k): v[0] for k, v in tuned.items()}},
      'refined_cells_per_s': cells / (min(graph, graph_tuned) * 1e-3),
      'refined_cells': cells,
      'rel_err_fp32_vs_fp64': rel,
      'checksum': float(ref.double().sum()),
      'steps': args.steps, 'warmup': args.warmup, 'dtype': 'f32', 'data': 'synthetic',
  }
  print(json.dumps(line))


# MMD^2 gradient workload (not the default bench line): 128 'generated' and
# 128 'target' Brownian paths with per-path drift ~ N(0, 0.5), L = 128,
# d = 4, SignaturePDEKernel(dyadic_order=2), RBF bandwidth 1.  Times
# MMD^2 = mean K(X,X) + mean K(Y,Y) - 2 mean K(X,Y) and its gradient with
# respect to X and the bandwidth (FP32), and checks the FP64 gradient against
# central finite differences (h = 1e-6) on 16 random coordinates.

def make_drift_paths(n, L, d, seed):
  rng = np.random.default_rng(seed)
  drift = rng.standard_normal((n, 1, d)) * np.sqrt(0.5)
  inc = rng.standard_normal((n, L - 1, d)) / np.sqrt(L) + drift / L
  return np.concatenate([np.zeros((n, 1, d)), np.cumsum(inc, 1)], 1)


def run_mmd_pde(args):
  import torch

  import ksig_b200 as K
  n = args.n_seq or 128
  dev = torch.device('cuda', 0)
  Xn = make_drift_paths(n, 128, 4, 41)
  Yn = make_drift_paths(n, 128, 4, 42)

  def mmd2(kern, X, Y):
    return (kern(X, return_on_gpu=True).mean() + kern(Y, return_on_gpu=True).mean()
            - 2.0 * kern(X, Y, return_on_gpu=True).mean())

  def timed(fn, steps, warm):
    for _ in range(warm):
      fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
      a = torch.cuda.Event(enable_timing=True)
      b = torch.cuda.Event(enable_timing=True)
      a.record()
      fn()
      b.record()
      b.synchronize()
      ts.append(a.elapsed_time(b))
    return sum(ts) / len(ts)

  X32 = torch.tensor(Xn, dtype=torch.float32, device=dev, requires_grad=True)
  Y32 = torch.tensor(Yn, dtype=torch.float32, device=dev)
  bw = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
  kern = K.SignaturePDEKernel(dyadic_order=2, static_kernel=K.RBFKernel(bw))

  def fwd():
    with torch.no_grad():
      mmd2(kern, X32, Y32)

  def fb():
    X32.grad = None
    bw.grad = None
    mmd2(kern, X32, Y32).backward()

  fwd_ms = timed(fwd, args.steps, args.warmup)
  fb_ms = timed(fb, args.steps, args.warmup)
  if args.no_cpu:  # skip the finite-difference check (profiling runs)
    fd = None
  else:
    X64 = torch.tensor(Xn, dtype=torch.float64, device=dev, requires_grad=True)
    Y64 = torch.tensor(Yn, dtype=torch.float64, device=dev)
    b64 = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    mmd2(K.SignaturePDEKernel(dyadic_order=2, static_kernel=K.RBFKernel(b64)),
         X64, Y64).backward()
    gX = X64.grad.cpu().numpy()

    def f(Xv, b):
      k = K.SignaturePDEKernel(dyadic_order=2, static_kernel=K.RBFKernel(b))
      with torch.no_grad():
        return float(mmd2(k, torch.tensor(Xv, device=dev), Y64))

    rng = np.random.default_rng(7)
    h = 1e-6
    errs = []
    for _ in range(16):
      i = tuple(int(rng.integers(0, s)) for s in Xn.shape)
      Xp, Xm = Xn.copy(), Xn.copy()
      Xp[i] += h
      Xm[i] -= h
      d_fd = (f(Xp, 1.0) - f(Xm, 1.0)) / (2 * h)
      errs.append(abs(d_fd - gX[i]) / max(np.abs(gX).max(), 1e-300))
    fdb = (f(Xn, 1.0 + h) - f(Xn, 1.0 - h)) / (2 * h)
    fd = {'coords': 16, 'h': h, 'max_rel_err_dX': float(max(errs)),
          'dbandwidth': float(b64.grad), 'dbandwidth_fd': fdb,
          'rel_err_dbandwidth': abs(fdb - float(b64.grad)) / max(1.0, abs(fdb))}
  line = {
      'metric': METRIC, 'workload': f'mmd2_sig_pde_rbf_N{n}_M{n}_L128_d4_dyadic2',
      'forward_ms': fwd_ms, 'fwd_bwd': {'s_per_step': fb_ms * 1e-3, 'ms_per_step': fb_ms,
                                        'what': 'MMD^2 and d/dX, d/dbandwidth (FP32)'},
      'fd_check_fp64': fd,
      'steps': args.steps, 'warmup': args.warmup, 'dtype': 'f32', 'data': 'synthetic',
  }
  print(json.dumps(line))


# ---------------------------------------------------------------------------
# Reference arm: the reference recursion on the host cores.
# ---------------------------------------------------------------------------

def _cupy_probe():
  """Whether the reference's own GPU path (CuPy) could run on this host."""
  try:
    import cupy  # noqa: F401
    return {'available': True, 'version': getattr(cupy, '__version__', '?')}
  except Exception as e:  # noqa: BLE001 - any import failure means unavailable
    return {'available': False, 'reason': f'{type(e).__name__}: {e}'[:200]}


def run_reference(args, rank, world):
  if rank != 0:
    return
  import multiprocessing as mp
  cores = os.cpu_count() or 1
  ctx = mp.get_context('spawn')
  n = args.ref_pairs
  with ctx.Pool(cores) as pool:
    for _ in range(args.warmup):
      cpu_sample(n, n, 7, pool)
    t = [cpu_sample(n, n, 7 + i, pool) for i in range(args.steps)]
  secs = sum(t) / len(t)
  value = n * n / secs
  line = {
      'metric': METRIC, 'value': value, 'unit': UNIT, 'impl': 'reference',
      'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
      'ms_per_step': secs * 1e3, 'higher_is_better': True, 'scaling': 'weak',
      'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
      'config': config(world),
      'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores,
                       'kind': 'port',
                       'sample': f'{n}x{n} pairs per step (+ diagonal passes) '
                                 'of the same workload; the reference needs '
                                 'CuPy on a GPU, so its recursion runs as the '
                                 'NumPy restatement in oracle/ over a '
                                 f'{cores}-process pool'},
      'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0,
              'd2h_bytes_per_step': 0},
      # The reference's CuPy path on the GPU needs CuPy, which this image
      # does not ship; the probe records why it is not timed.
      'reference_cupy_path': _cupy_probe(),
  }
  print(json.dumps(line))


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--gpus', type=int, default=1)
  ap.add_argument('--steps', type=int, default=20)
  ap.add_argument('--warmup', type=int, default=5)
  ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
  ap.add_argument('--cpu-pairs', type=int, default=40)
  ap.add_argument('--ref-pairs', type=int, default=32)
  ap.add_argument('--no-cpu', action='store_true')
  ap.add_argument('--no-bwd', action='store_true')
  ap.add_argument('--no-plain', action='store_true')
  ap.add_argument('--no-ragged', action='store_true',
                  help='skip the ragged order-2 sub-record of the bench line')
  ap.add_argument('--bwd-steps', type=int, default=10)
  ap.add_argument('--workload', default='dp512',
                  choices=['dp512', 'ragged-dp', 'ragged-pde', 'mmd-pde', 'gram-forms'],
                  help='dp512: the bench line; ragged-dp: the 2048 x 2048 ragged '
                       'order-2 workload, printed as its own report line')
  ap.add_argument('--plain-sample', type=int, default=96)
  ap.add_argument('--gram-d', default=None,
                  help='gram-forms: comma-separated channel counts (with time)')
  ap.add_argument('--gram-forms', default=None,
                  help='gram-forms: comma-separated subset of register,tensor,cuda')
  ap.add_argument('--n-seq', type=int, default=None,
                  help='sequences per side; smaller values are for profiling '
                       'captures only, not bench lines')
  args = ap.parse_args()
  if args.n_seq is not None and args.workload == 'dp512':
    globals()['N_SEQ'] = args.n_seq
  args.warmup = max(args.warmup, 3)
  world = int(os.environ.get('WORLD_SIZE', '1'))
  rank = int(os.environ.get('RANK', '0'))
  if args.impl == 'reference':
    run_reference(args, rank, world)
    return
  import torch
  dist = None
  if world > 1:
    import datetime
    import torch.distributed as tdist
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    tdist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    dist = tdist
  else:
    torch.cuda.set_device(0)
  if args.workload == 'ragged-dp':
    run_ragged(args)
    return
  if args.workload == 'ragged-pde':
    run_ragged_pde(args)
    return
  if args.workload == 'mmd-pde':
    run_mmd_pde(args)
    return
  if args.workload == 'gram-forms':
    run_gram_forms(args)
    return
  try:
    run_ours(args, rank, world, dist)
  finally:
    if dist is not None:
      dist.barrier()
      dist.destroy_process_group()


if __name__ == '__main__':
  main()
