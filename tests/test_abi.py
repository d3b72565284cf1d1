"""The C ABI without a GPU: every declared symbol is exported, the ctypes
mirrors match the C struct layouts, and argument errors are reported
before any CUDA call."""
import ctypes
import os
import re
import subprocess

import pytest

from hlld_ai_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hlld_b200.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(hlld_\w+)\(", src, re.M)))


def test_header_declares_the_plugin_and_step_entry_points():
    names = declared_functions()
    for need in ("hlld_riemann_faces", "hlld_cons_to_prim", "hlld_prim_to_cons",
                 "hlld_rk_step_ct", "hlld_sync_state", "hlld_compute_dt_2d", "hlld_sweep2d",
                 "hlld_ct_update2d", "hlld_step2d_scratch_bytes"):
        assert need in names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for name in declared_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (hlld_\w+)$", out, re.M))
    assert set(declared_functions()) <= exported
    assert set(_lib.SIGNATURES) <= exported


PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "hlld_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(hlld_flux_diag_t), sizeof(hlld_step_diag_t),
         sizeof(hlld_grid2d_t), sizeof(hlld_state2d_t), sizeof(hlld_tubes_t));
  printf("%zu %zu %zu %zu %zu\n", offsetof(hlld_grid2d_t, dx), offsetof(hlld_grid2d_t, gamma),
         offsetof(hlld_grid2d_t, upwind), offsetof(hlld_state2d_t, Bxf),
         offsetof(hlld_step_diag_t, speed_max_bits));
  return 0;
}
"""


def test_struct_layouts_match_ctypes(tmp_path):
    c = tmp_path / "probe.c"
    c.write_text(PROBE)
    exe = tmp_path / "probe"
    cc = "x86_64-linux-gnu-gcc-13" if subprocess.run(["which", "x86_64-linux-gnu-gcc-13"],
                                                      capture_output=True).returncode == 0 else "gcc"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(x) for x in out[:5]]
    offs = [int(x) for x in out[5:]]
    assert sizes == [ctypes.sizeof(_lib.FluxDiag), ctypes.sizeof(_lib.StepDiag),
                     ctypes.sizeof(_lib.Grid2DC), ctypes.sizeof(_lib.State2DC),
                     ctypes.sizeof(_lib.TubesC)]
    assert offs == [_lib.Grid2DC.dx.offset, _lib.Grid2DC.gamma.offset, _lib.Grid2DC.upwind.offset,
                    _lib.State2DC.Bxf.offset, _lib.StepDiag.speed_max_bits.offset]


def grid(**kw):
    base = dict(nx=64, ny=64, ng=2, dx=1 / 64, dy=1 / 64, bc_x=0, bc_y=1, limiter=1, solver=1,
                gamma=5 / 3, atmo_rho=1e-10, upwind=1, precision=0)
    base.update(kw)
    return _lib.Grid2DC(**base)


def test_scratch_size_and_argument_errors_without_gpu():
    L = _lib.lib()
    n = ctypes.c_size_t(0)
    g = grid()
    assert L.hlld_step2d_scratch_bytes(ctypes.byref(g), ctypes.byref(n)) == 0
    nxt = 68
    assert n.value >= 8 * (7 * 2 * (nxt + 1) * nxt + 6 * nxt * nxt)
    for bad in (dict(ng=1, limiter=3), dict(nx=2), dict(bc_x=5), dict(solver=7),
                dict(gamma=1.0), dict(limiter=9), dict(dx=0.0), dict(emf_mode=2)):
        gb = grid(**bad)
        rc = L.hlld_step2d_scratch_bytes(ctypes.byref(gb), ctypes.byref(n))
        assert rc == _lib.HLLD_OK - 1, bad  # HLLD_ERR_INVALID
        assert L.hlld_last_error_detail()
    # the adjoint takes the solver's face EMF only
    ta, sa = ctypes.c_size_t(0), ctypes.c_size_t(0)
    gh = grid(emf_mode=1)
    assert L.hlld_step2d_scratch_bytes(ctypes.byref(gh), ctypes.byref(n)) == 0
    assert L.hlld_adjoint_tape_bytes(ctypes.byref(gh), ctypes.byref(ta), ctypes.byref(sa)) == -3
    gm = grid(precision=9)
    assert L.hlld_step2d_scratch_bytes(ctypes.byref(gm), ctypes.byref(n)) == -3
    s = _lib.State2DC()
    # NULL state arrays and NULL scratch are rejected on the host
    assert L.hlld_rk_step_ct(ctypes.byref(g), ctypes.byref(s), None, 0, 1e-3, None, 3, None,
                             None) == -1
    assert L.hlld_riemann_faces(10, None, None, 0, 1, 5 / 3, 0, None, None, None, None, None,
                                None, None, None) == -1
    assert L.hlld_cons_to_prim(10, None, 5 / 3, 1e-10, 1e-10, 0, None, None, None) == -1
    assert L.hlld_error_string(-4) == b"scratch buffer too small"
    # the C2P start from the primitives belongs to the mixed form: a NULL state
    # and an FP64 grid are refused on the host (the non-NULL addresses of the
    # second state are never dereferenced)
    assert L.hlld_sync_state_from_prims(ctypes.byref(g), ctypes.byref(s), None, None, None,
                                        None) == -1
    fake = _lib.State2DC()
    for k in range(6):
        fake.cons[k] = 256
    for k in range(9):
        fake.prims[k] = 256
    fake.Bxf = fake.Byf = 256
    assert L.hlld_sync_state_from_prims(ctypes.byref(grid(precision=0)), ctypes.byref(fake), None,
                                        None, None, None) == -3


def test_tube_batch_argument_errors_without_gpu():
    L = _lib.lib()
    empty = _lib.TubesC(ntubes=0, ng=3, cfl=0.4, tend=0.1, limiter=3, solver=1, scheme=3,
                        gamma=5 / 3)
    assert L.hlld_tubes_run(ctypes.byref(empty), None, None, None, None, None, None, None, 0, 0,
                            None) == 0
    b = _lib.TubesC(ntubes=4, ng=3, cfl=0.4, tend=0.1, limiter=3, solver=1, scheme=3, gamma=5 / 3)
    assert L.hlld_tubes_run(ctypes.byref(b), None, None, None, None, None, None, None, 0, 0,
                            None) == -1
    assert L.hlld_tubes_run(None, None, None, None, None, None, None, None, 0, 0, None) == -1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError):
        _lib.lib()
