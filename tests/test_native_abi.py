"""CPU: the C-ABI library loads, exports every declared symbol, and its
struct layouts match the ctypes mirror (no kernel is launched)."""

import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from swirlc_b200 import _native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'swirlc_b200.h')


def _declared():
  with open(HEADER) as f:
    text = f.read()
  return sorted(set(re.findall(r'\b(swc_\w+)\s*\(', text)))


@pytest.fixture(scope='module')
def lib():
  if not os.path.exists(nat.lib_path()):
    from swirlc_b200 import build
    build.build()
  return nat.load(require_cuda=False)


def test_every_declared_symbol_is_exported(lib):
  names = _declared()
  assert set(names) == set(nat.EXPORTED)
  for name in names:
    assert hasattr(lib, name), name


def test_abi_version_and_error_buffer(lib):
  assert lib.swc_abi_version() == 1
  buf = ctypes.create_string_buffer(64)
  assert lib.swc_last_error(buf, len(buf)) >= 0


def test_argument_errors_need_no_gpu(lib):
  # Validation runs before any CUDA call and maps to ValueError.
  with pytest.raises(ValueError):
    nat.check(lib.swc_rk_stage(None, None, None, None, None, 0, 0.0, 0.0,
                               None, None, None))
  with pytest.raises(ValueError):
    nat.check(lib.swc_clock_begin_step(None, None))
  with pytest.raises(ValueError):
    nat.check(lib.swc_rk_step_noalloc(None, None, None, 3, None, None, None))
  with pytest.raises(ValueError):
    nat.check(lib.swc_batch_step(None, 3, 1, None, None))
  with pytest.raises(ValueError):
    nat.check(lib.swc_rk_stage_ext(None, None, None, None, None, None, 0, 0.0,
                                   0.0, None, None, None))


def test_step_vjp_argument_errors_need_no_gpu(lib):
  # Order and aliasing checks run before any CUDA call; the pointers are
  # only compared, never dereferenced.
  def arr(lo, hi):
    return (ctypes.c_void_p * (hi - lo))(*[0x10000 + 256 * i
                                          for i in range(lo, hi)])
  stages, g, work = arr(0, 15), arr(15, 20), arr(20, 30)
  gn, scratch = arr(30, 35), arr(35, 40)
  with pytest.raises(NotImplementedError):
    nat.check(lib.swc_rk_step_vjp(None, None, None, 4, stages, 1e-3, g, gn,
                                  work, None, scratch, None))
  for bad in (arr(10, 15), arr(15, 20), arr(25, 30)):  # a stage, g, work
    with pytest.raises(ValueError):
      nat.check(lib.swc_rk_step_vjp(None, None, None, 3, stages, 1e-3, g, bad,
                                    work, None, scratch, None))
  # RK2: gn must not alias g1 (work[0:5]) either.
  with pytest.raises(ValueError):
    nat.check(lib.swc_rk_step_vjp(None, None, None, 2, stages, 1e-3, g,
                                  arr(20, 25), work, None, scratch, None))


def test_noalloc_limit_matches_header():
  with open(os.path.join(ROOT, 'include', 'swirlc_b200.h')) as f:
    text = f.read()
  m = re.search(r'#define SWC_NOALLOC_MAX_BYTES \((\d+)ll << (\d+)\)', text)
  assert m and int(m.group(1)) << int(m.group(2)) == nat.SWC_NOALLOC_MAX_BYTES


def test_header_constants_match_python():
  with open(os.path.join(ROOT, 'include', 'swirlc_b200.h')) as f:
    text = f.read()
  for name in ('SWC_VJP_SCRATCH', 'SWC_MAX_OVERRIDES', 'SWC_MAX_FIELDS'):
    m = re.search(r'#define %s (\d+)' % name, text)
    assert m and int(m.group(1)) == getattr(nat, name), name


def _c_layout():
  src = r'''
#include <stddef.h>
#include <stdio.h>
#include "swirlc_b200.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m));
int main(void) {
  printf("SwcGrid %zu\n", sizeof(SwcGrid));
  printf("SwcScheme %zu\n", sizeof(SwcScheme));
  printf("SwcBC %zu\n", sizeof(SwcBC));
  printf("SwcFieldBC %zu\n", sizeof(SwcFieldBC));
  printf("SwcClock %zu\n", sizeof(SwcClock));
  printf("SwcBatchMember %zu\n", sizeof(SwcBatchMember));
  printf("SwcOverride %zu\n", sizeof(SwcOverride));
  printf("SwcStageExt %zu\n", sizeof(SwcStageExt));
  F(SwcGrid, sx) F(SwcGrid, dz) F(SwcScheme, nu) F(SwcScheme, g)
  F(SwcScheme, pe_axis) F(SwcScheme, zseg) F(SwcBC, value) F(SwcBC, planes)
  F(SwcFieldBC, side) F(SwcClock, step)
  F(SwcBatchMember, u) F(SwcBatchMember, work) F(SwcBatchMember, pe_axis)
  F(SwcBatchMember, bcs) F(SwcBatchMember, clock) F(SwcBatchMember, tile)
  F(SwcBatchMember, zseg)
  F(SwcOverride, value) F(SwcOverride, plane) F(SwcStageExt, boundary)
  F(SwcStageExt, nface) F(SwcStageExt, nflux) F(SwcStageExt, face)
  F(SwcStageExt, flux)
  return 0;
}
'''
  with tempfile.TemporaryDirectory() as d:
    c = os.path.join(d, 'layout.c')
    exe = os.path.join(d, 'layout')
    with open(c, 'w') as f:
      f.write(src)
    subprocess.run(['gcc', '-I', os.path.join(ROOT, 'include'), c, '-o', exe],
                   check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True)
  return dict(line.rsplit(' ', 1) for line in out.stdout.strip().splitlines())


def test_struct_layouts_match_header():
  c = {k: int(v) for k, v in _c_layout().items()}
  assert c['SwcGrid'] == ctypes.sizeof(nat.SwcGrid)
  assert c['SwcScheme'] == ctypes.sizeof(nat.SwcScheme)
  assert c['SwcBC'] == ctypes.sizeof(nat.SwcBC)
  assert c['SwcFieldBC'] == ctypes.sizeof(nat.SwcFieldBC)
  assert c['SwcClock'] == ctypes.sizeof(nat.SwcClock)
  assert c['SwcBatchMember'] == ctypes.sizeof(nat.SwcBatchMember)
  assert c['SwcOverride'] == ctypes.sizeof(nat.SwcOverride)
  assert c['SwcStageExt'] == ctypes.sizeof(nat.SwcStageExt)
  for key, off in c.items():
    if '.' not in key:
      continue
    st, field = key.split('.')
    assert getattr(getattr(nat, st), field).offset == off, key
