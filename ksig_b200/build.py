"""Builds ``ksig_b200/lib/libksig_b200.so`` (sm_100a) in-tree with nvcc.

The hot kernels are templates over the compute type, the padded point
dimension KD, the columns per lane C, the number of levels NL and the order
P (or the dyadic refinement F for the PDE).  This script writes one
translation unit per group of instantiations under ``csrc/gen/`` together
with a registry table the C ABI searches at run time, compiles the units in
parallel and links the shared library.  Rebuilds are incremental (object
files newer than every source they depend on are kept).

    python -m ksig_b200.build [-j N] [--force]
"""

import argparse
import concurrent.futures as cf
import itertools
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
GEN = os.path.join(CSRC, 'gen')
OBJ = os.path.join(HERE, '_build')
LIB_DIR = os.path.join(HERE, 'lib')
LIB = os.path.join(LIB_DIR, 'libksig_b200.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ['-O3', '-std=c++17', '-Xcompiler', '-fPIC',
              '-Xcompiler', '-O2', '--expt-relaxed-constexpr', '-ftz=true']
# Line info (source correlation for ncu) on the C ABI and the FP32 order-1
# DP forward units (the profiled sweeps); the other units are built without
# it, which keeps the library about half its size (line info makes a unit's
# object 3.7 times larger).
def _wants_lineinfo(src):
  name = os.path.basename(src)
  return name == 'capi.cu' or name.startswith('inst_dp_f32_p1_d1_')
WPB = 2  # warps per block of the sweep kernels

KD_ALL = [2, 4, 6, 8, 9, 10, 12, 16, 24, 32]
KD_MID = [2, 4, 8, 9, 12, 16, 32]
KD_FEW = [4, 8, 16, 32]
NL_ALL = [1, 2, 3, 4, 5, 6, 8]


def instances():
  """(op, dtype, kd, c, nl, p, diff) tuples.  op: dp/pde/dpb/pdeb."""
  out = []
  add = out.append
  # DP forward, float.  No 7-column tiles above 16 coordinates: there the
  # column points no longer fit in registers (tens of KB of spills per
  # thread; 2.6x to 11x slower than 4 columns at L = 200 on B200).
  for nl, kd, c in itertools.product(NL_ALL, KD_ALL, [2, 4, 7]):
    if c < 7 or kd <= 16:
      add(('dp', 'f32', kd, c, nl, 1, 1))
  for nl, kd, c in itertools.product([2, 3, 4, 5, 6, 8], KD_ALL, [2, 4]):
    add(('dp', 'f32', kd, c, nl, 2, 1))
  for p, nls in ((3, [3, 4, 5, 6, 8]), (4, [4, 5, 6, 8])):
    for nl, kd in itertools.product(nls, KD_FEW):
      add(('dp', 'f32', kd, 2, nl, p, 1))
  for p, nls in ((1, NL_ALL), (2, [2, 3, 4, 5, 6, 8])):
    for nl, kd in itertools.product(nls, KD_FEW):
      add(('dp', 'f32', kd, 2, nl, p, 0))
  # DP forward, double.
  for p, nls, kds in ((1, NL_ALL, KD_MID), (2, [2, 3, 4, 5, 6, 8], KD_FEW),
                      (3, [3, 4, 5, 6, 8], KD_FEW), (4, [4, 5, 6, 8], KD_FEW)):
    for nl, kd in itertools.product(nls, kds):
      add(('dp', 'f64', kd, 2, nl, p, 1))
  for p, nls in ((1, NL_ALL), (2, [2, 3, 4, 5, 6, 8])):
    for nl, kd in itertools.product(nls, KD_FEW):
      add(('dp', 'f64', kd, 2, nl, p, 0))
  # PDE forward.  8-column tiles up to 16 coordinates only (beyond, they
  # spill: 5x to 17x slower than 4 columns at d = 24 and 32 on B200).
  for f, kd, c in itertools.product([1, 2, 4, 8], KD_ALL, [2, 4, 8]):
    if c < 8 or kd <= 16:
      add(('pde', 'f32', kd, c, 0, f, 1))
  for f, kd in itertools.product([1, 2, 4, 8], KD_MID):
    add(('pde', 'f64', kd, 2, 0, f, 1))
  for dt in ('f32', 'f64'):
    for f, kd in itertools.product([1, 2, 4], KD_FEW):
      add(('pde', dt, kd, 2, 0, f, 0))
  # Forward sweeps for the other static kernels (polynomial, Matern,
  # rational quadratic): one tile width per dtype.
  for dt, c in (('f32', 4), ('f64', 2)):
    for p, nls in ((1, NL_ALL), (2, [2, 3, 4, 5, 6, 8])):
      for nl, kd in itertools.product(nls, KD_FEW):
        add(('dpx', dt, kd, c, nl, p, 1))
    for f, kd in itertools.product([1, 2, 4, 8], KD_FEW):
      add(('pdex', dt, kd, c, 0, f, 1))
  # Global alignment kernel (no differencing).
  for kd, c in itertools.product(KD_ALL, [2, 4, 8]):
    if c < 8 or kd <= 16:  # same register limit as the PDE forward
      add(('ga', 'f32', kd, c, 0, 1, 0))
  for kd in KD_MID:
    add(('ga', 'f64', kd, 2, 0, 1, 0))
  # PDE backward (row-side gradients).
  # The adjoint keeps three C*F-wide rows in registers: C*F <= 16, and
  # 8-column tiles up to 12 coordinates (4 columns are 1.2x faster at
  # d = 16 and 5.7x faster at d = 32 on B200).
  for f, kd, c in itertools.product([1, 2, 4, 8], KD_MID, [2, 4, 8]):
    if c * f <= 16 and (c < 8 or kd <= 12):
      add(('pdeb', 'f32', kd, c, 0, f, 1))
  for f, kd in itertools.product([1, 2, 4, 8], KD_FEW):
    add(('pdeb', 'f64', kd, 2, 0, f, 1))
  # Deep truncations (n_levels 10 and 12, order 1): the narrower tiles only,
  # since the per-level column sums grow the register state.
  for nl, kd, c in itertools.product([10, 12], KD_MID, [2, 4]):
    add(('dp', 'f32', kd, c, nl, 1, 1))
  for nl, kd in itertools.product([10, 12], KD_FEW):
    add(('dp', 'f64', kd, 2, nl, 1, 1))
    add(('dpb', 'f64', kd, 2, nl, 1, 1))
  for nl, kd, c in itertools.product([10, 12], KD_MID, [2, 4]):
    if c < 4 or kd <= 16:
      add(('dpb', 'f32', kd, c, nl, 1, 1))
  # DP backward (row-side gradients).  The adjoint holds more per-column
  # state than the forward: 7-column tiles only up to 12 coordinates and
  # 4-column tiles up to 16 (beyond that they spill heavily; measured on
  # B200, d = 16: 4 columns 1.1-1.6x faster than 7; d = 32: 2 columns 1.7x
  # faster than 4 and 13x faster than 7).
  for dt, cs, kds in (('f32', [2, 4, 7], KD_MID), ('f64', [2], KD_FEW)):
    for nl, kd, c in itertools.product(NL_ALL, kds, cs):
      if c == 2 or (c == 4 and kd <= 16) or (c == 7 and kd <= 12):
        add(('dpb', dt, kd, c, nl, 1, 1))
    for nl, kd in itertools.product([2, 3, 4, 5, 6, 8], kds):
      add(('dpb', dt, kd, 2, nl, 2, 1))
      if dt == 'f32' and kd in KD_FEW:
        add(('dpb', dt, kd, 3, nl, 2, 1))  # wider order-2 strips
    for p, nls in ((3, [3, 4, 5, 6, 8]), (4, [4, 5, 6, 8])):
      for nl, kd in itertools.product(nls, KD_FEW):
        add(('dpb', dt, kd, 2, nl, p, 1))
  # Orders 5 to 8 (order 0 = full order up to n_levels 8), forward and
  # adjoint: the narrowest tile only (the level states grow as p^2).
  for dt in ('f32', 'f64'):
    for p in (5, 6, 7, 8):
      for nl, kd in itertools.product([nl for nl in (5, 6, 8) if nl >= p], KD_FEW):
        add(('dp', dt, kd, 2, nl, p, 1))
        add(('dpb', dt, kd, 2, nl, p, 1))
  # Deeper truncations: order 1 up to 32 levels, order 2 up to 16.
  for dt in ('f32', 'f64'):
    for (p, nl), kd in itertools.product(
        [(1, 16), (1, 20), (1, 24), (1, 32), (2, 10), (2, 12), (2, 16)], KD_FEW):
      add(('dp', dt, kd, 2, nl, p, 1))
      add(('dpb', dt, kd, 2, nl, p, 1))
  # Gram-input forward sweeps (kd = 0, gram.cuh): every channel count and
  # static kind, for the shapes the register-Gram tiles do not cover.
  for dt in ('f32', 'f64'):
    wide = [2, 4, 7] if dt == 'f32' else [2]
    for nl, c in itertools.product(NL_ALL + [10, 12, 16, 20, 24, 32], wide):
      add(('dp', dt, 0, c, nl, 1, 1))
    for nl, c in itertools.product([2, 3, 4, 5, 6, 8, 10, 12, 16], wide[:2]):
      add(('dp', dt, 0, c, nl, 2, 1))
    for p in (3, 4, 5, 6, 7, 8):
      for nl in (3, 4, 5, 6, 8):
        if nl >= p:
          add(('dp', dt, 0, 2, nl, p, 1))
    for p, nls in ((1, NL_ALL), (2, [2, 3, 4, 5, 6, 8])):
      for nl in nls:
        add(('dp', dt, 0, 2, nl, p, 0))
    for f, c in itertools.product([1, 2, 4, 8], [2, 4, 8] if dt == 'f32' else [2]):
      add(('pde', dt, 0, c, 0, f, 1))
    for f in (1, 2, 4):
      add(('pde', dt, 0, 2, 0, f, 0))
    for c in ([2, 4, 8] if dt == 'f32' else [2]):
      add(('ga', dt, 0, c, 0, 1, 0))
  # The adjoint with strip checkpointing: one per adjoint tile.
  out += [('dpc',) + inst[1:] for inst in out if inst[0] == 'dpb']
  # Forward pass of the split gradient pass: one per order-1 adjoint tile
  # with at least two levels (same tile, same records).
  out += [('dpr',) + inst[1:] for inst in out
          if inst[0] == 'dpb' and inst[5] == 1 and inst[4] >= 2]
  # PDE forward with stacked pairs (equal-length full grids), for the tiles
  # the sweep stacks (differencing, up to 12 coordinates).
  out += [('pdes',) + inst[1:] for inst in out
          if inst[0] == 'pde' and inst[6] == 1 and 0 < inst[2] <= 12]
  return out


OPS = {
    'dp': ('OP_DP_FWD', 'dp_fwd_kernel<{T}, {kd}, {c}, {nl}, {p}, {diff}, {wpb}, false>'),
    'pde': ('OP_PDE_FWD', 'pde_fwd_kernel<{T}, {kd}, {c}, {p}, {diff}, {wpb}, false>'),
    'dpx': ('OP_DP_FWD_EXT', 'dp_fwd_kernel<{T}, {kd}, {c}, {nl}, {p}, {diff}, {wpb}, true>'),
    'pdex': ('OP_PDE_FWD_EXT', 'pde_fwd_kernel<{T}, {kd}, {c}, {p}, {diff}, {wpb}, true>'),
    'pdes': ('OP_PDE_FWD_STACK', 'pde_fwd_kernel<{T}, {kd}, {c}, {p}, {diff}, {wpb}, false, true>'),
    'ga': ('OP_GA_FWD', 'ga_fwd_kernel<{T}, {kd}, {c}, {wpb}>'),
    'dpb': ('OP_DP_BWD', 'dp_bwd_kernel<{T}, {kd}, {c}, {nl}, {p}, {wpb}>'),
    'dpr': ('OP_DP_REC_FWD', 'dp_rec_fwd_kernel<{T}, {kd}, {c}, {nl}, {p}, {wpb}>'),
    'dpc': ('OP_DP_BWD_CKPT', 'dp_bwd_ckpt_kernel<{T}, {kd}, {c}, {nl}, {p}, {wpb}>'),
    'pdeb': ('OP_PDE_BWD', 'pde_bwd_kernel<{T}, {kd}, {c}, {p}, {wpb}>'),
}


HEADER = {'dp': 'sweep.cuh', 'pde': 'sweep.cuh', 'dpx': 'sweep.cuh',
          'pdex': 'sweep.cuh', 'pdes': 'sweep.cuh', 'ga': 'sweep.cuh', 'dpb': 'dp_bwd.cuh',
          'dpr': 'dp_bwd.cuh', 'dpc': 'dp_bwd.cuh', 'pdeb': 'pde_bwd.cuh'}


def _group_key(inst):
  op, dt, kd, c, nl, p, diff = inst
  return f'{op}_{dt}_p{p}_d{diff}_kd{kd}'


def generate():
  """Writes csrc/gen/*.cu; returns the list of generated unit paths."""
  os.makedirs(GEN, exist_ok=True)
  groups = {}
  for inst in instances():
    groups.setdefault(_group_key(inst), []).append(inst)
  units = []
  tables = []
  for key, insts in sorted(groups.items()):
    # Each unit includes only the header of its kernel family, so that an
    # edit to one family's header rebuilds only that family.
    lines = ['// Generated by ksig_b200/build.py; do not edit.',
             f'#include "../{HEADER[insts[0][0]]}"',
             '#include "../registry.h"',
             'namespace ksig {']
    ents = []
    for op, dt, kd, c, nl, p, diff in insts:
      T = 'float' if dt == 'f32' else 'double'
      opname, tmpl = OPS[op]
      name = tmpl.format(T=T, kd=kd, c=c, nl=nl, p=p,
                         diff='true' if diff else 'false', wpb=WPB)
      ents.append(f'  {{{opname}, {int(dt == "f64")}, {kd}, {c}, {nl}, {p}, '
                  f'{diff}, {WPB}, (const void*)&{name}}},')
    lines.append(f'extern const KernelEntry kTab_{key}[] = {{')
    lines += ents
    lines.append('};')
    lines.append(f'extern const int kTabN_{key} = {len(ents)};')
    lines.append('}  // namespace ksig')
    path = os.path.join(GEN, f'inst_{key}.cu')
    _write_if_changed(path, '\n'.join(lines) + '\n')
    units.append(path)
    tables.append(key)
  reg = ['// Generated by ksig_b200/build.py; do not edit.',
         '#include "../registry.h"', 'namespace ksig {']
  for key in tables:
    reg.append(f'extern const KernelEntry kTab_{key}[];')
    reg.append(f'extern const int kTabN_{key};')
  reg.append('const KernelTable kAllTables[] = {')
  for key in tables:
    reg.append(f'  {{kTab_{key}, {len(groups[key])}}},')
  reg.append('};')
  reg.append(f'const int kNumTables = {len(tables)};')
  reg.append('}  // namespace ksig')
  path = os.path.join(GEN, 'registry_tables.cu')
  _write_if_changed(path, '\n'.join(reg) + '\n')
  units.append(path)
  return units


def _write_if_changed(path, text):
  if os.path.exists(path):
    with open(path) as f:
      if f.read() == text:
        return
  with open(path, 'w') as f:
    f.write(text)


_INC_CACHE = {}


def _includes(path):
  """Files a source includes with #include "...", transitively."""
  path = os.path.normpath(path)
  if path in _INC_CACHE:
    return _INC_CACHE[path]
  _INC_CACHE[path] = set()
  out = set()
  try:
    with open(path) as f:
      text = f.read()
  except OSError:
    return out
  for line in text.splitlines():
    line = line.strip()
    if line.startswith('#include "'):
      inc = os.path.normpath(os.path.join(os.path.dirname(path), line.split('"')[1]))
      if os.path.exists(inc):
        out.add(inc)
        out |= _includes(inc)
  _INC_CACHE[path] = out
  return out


def _nvcc():
  cand = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
  return cand


def _compile(src, obj, force):
  deps = [src] + sorted(_includes(src)) + [os.path.abspath(__file__)]
  if (not force and os.path.exists(obj)
      and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps)):
    return obj, None
  cmd = [_nvcc()] + ARCH + NVCC_FLAGS + (['-lineinfo'] if _wants_lineinfo(src) else []) + [
      '-I', os.path.join(ROOT, 'include'), '-c', src, '-o', obj]
  r = subprocess.run(cmd, capture_output=True, text=True)
  if r.returncode != 0:
    return obj, f'{" ".join(cmd)}\n{r.stdout}\n{r.stderr}'
  return obj, None


def build(jobs=None, force=False, verbose=True):
  units = generate()
  units = [os.path.join(CSRC, 'capi.cu')] + units
  os.makedirs(OBJ, exist_ok=True)
  os.makedirs(LIB_DIR, exist_ok=True)
  objs = []
  jobs = jobs or os.cpu_count() or 4
  errors = []
  with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
    futs = []
    for u in units:
      obj = os.path.join(OBJ, os.path.basename(u)[:-3] + '.o')
      objs.append(obj)
      futs.append(ex.submit(_compile, u, obj, force))
    for f in futs:
      _, err = f.result()
      if err:
        errors.append(err)
  if errors:
    raise RuntimeError('nvcc failed:\n' + '\n'.join(errors[:3]))
  if (force or not os.path.exists(LIB)
      or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
    cmd = [_nvcc()] + ARCH + ['-shared', '-o', LIB] + objs + ['-lcudart']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
      raise RuntimeError(f'link failed: {r.stdout}\n{r.stderr}')
  if verbose:
    print(f'built {LIB} ({len(instances())} kernel instantiations, '
          f'{len(units)} units)')
  return LIB


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('-j', type=int, default=None)
  ap.add_argument('--force', action='store_true')
  a = ap.parse_args()
  build(jobs=a.j, force=a.force)


if __name__ == '__main__':
  sys.exit(main())
