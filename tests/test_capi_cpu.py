"""CPU: the C-ABI library loads and exports every symbol include/stgipc.h declares; calls
that need no GPU behave (defaults, no-device error)."""
import ctypes as C
import os
import subprocess

import pytest

from conftest import ROOT, have_gpu


@pytest.fixture(scope="module")
def L():
    from stgipc import _lib
    if not os.path.exists(_lib.LIB_PATH):
        import importlib.util
        spec = importlib.util.spec_from_file_location("stg_build", os.path.join(ROOT, "stiff-gipc_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    return _lib.lib()


def test_exports_every_header_symbol(L):
    from stgipc import _lib
    syms = _lib.header_symbols()
    assert len(syms) >= 14
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    for s in syms:
        assert hasattr(L, s)


def test_config_default(L):
    from stgipc import _lib
    c = _lib.Config()
    L.stg_config_default(C.byref(c))
    assert c.bank_size == 16 and c.tol == 1e-4 and abs(c.max_iter_ratio - 0.3) < 1e-15
    assert c.precision == 0 and c.preconditioner == 1 and c.stop_rule == 0


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_create_without_device_reports_error(L):
    from stgipc import _lib
    h = C.c_void_p()
    c = _lib.Config()
    L.stg_config_default(C.byref(c))
    assert L.stg_create(C.byref(c), C.byref(h)) == _lib.STG_ERR_NO_DEVICE
    assert b"device" in L.stg_last_error()


def test_invalid_config_rejected_before_device(L):
    from stgipc import _lib
    h = C.c_void_p()
    c = _lib.Config()
    L.stg_config_default(C.byref(c))
    c.bank_size = 24
    assert L.stg_create(C.byref(c), C.byref(h)) == _lib.STG_ERR_INVALID
    assert L.stg_destroy(None) == _lib.STG_OK
    assert L.stg_convert(None, 0, None, None, None, None) == _lib.STG_ERR_INVALID


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from stgipc import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libstgipc.so"))
    with pytest.raises(ImportError):
        _lib.lib()


def test_learned_flag_validated_before_device(L):
    """The learned coarse correction needs MAS and a host or graph loop; other values and
    combinations are errors before any device work, not a silent plain solve."""
    from stgipc import _lib
    h = C.c_void_p()
    for learned, pre, loop in ((2, _lib.PRECOND["mas"], _lib.LOOP["graph"]),
                               (1, _lib.PRECOND["diag"], _lib.LOOP["graph"]),
                               (1, _lib.PRECOND["mas"], _lib.LOOP["persistent"])):
        c = _lib.Config()
        L.stg_config_default(C.byref(c))
        c.learned, c.preconditioner, c.loop_mode = learned, pre, loop
        assert L.stg_create(C.byref(c), C.byref(h)) == _lib.STG_ERR_INVALID
        assert b"learned" in L.stg_last_error()


def test_net_training_entry_points_validate(L):
    """stg_net_* handle-free calls reject bad arguments without touching a device."""
    from stgipc import _lib
    assert L.stg_net_scratch_bytes(0, 1) == 0
    assert L.stg_net_scratch_bytes(100, 2) > 0
    assert L.stg_net_train_step(None, None, None, 1, None, None, None, None, 1, 0.0, None, None, 0, None) == \
        _lib.STG_ERR_INVALID
    g = _lib.NetGraphC()
    assert L.stg_net_forward(C.byref(g), None, None, 1, None, None, None, 0, None) == _lib.STG_ERR_INVALID
    assert L.stg_net_configure(None, 1) == _lib.STG_ERR_INVALID


def test_header_compiles_as_c_and_links(L, tmp_path):
    """A C caller (the form a cgo / FFI binding takes): include/stgipc.h compiles as C99,
    every declared entry point resolves when linking against libstgipc.so, and the calls that
    need no device behave."""
    from stgipc import _lib
    syms = _lib.header_symbols()
    refs = "\n".join(f"    (void*)&{s}," for s in syms)
    src = tmp_path / "caller.c"
    src.write_text(f"""
#include <stdio.h>
#include "stgipc.h"
static void* table[] = {{
{refs}
}};
int main(void)
{{
    stg_config c;
    stg_config_default(&c);
    stg_handle h = 0;
    const int st = stg_create(&c, &h);
    const size_t nb = stg_net_scratch_bytes(100, 2), fb = stg_fem_scratch_bytes(10, 4);
    const int bad = stg_fem_newton_system(0, 0, 0, 0, 0, 0, 0, 0, 0.3, 1000, 0.01, -9.8, 0, 0, 0, 0, 0, 0, 0, 0, 0);
    printf("%d %d %d %d %d %d\\n", (int)(sizeof(table) / sizeof(table[0])), c.bank_size, st,
           nb > 0, fb > 0, bad);
    return 0;
}}
""")
    exe = tmp_path / "caller"
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                         str(exe), "-L", lib_dir, "-lstgipc", f"-Wl,-rpath,{lib_dir}"], capture_output=True, text=True)
    if cc.returncode != 0 and "cannot find -lstgipc" in cc.stderr:
        # the library is named libstgipc.so in-tree: link it by path
        cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                             str(exe), _lib.LIB_PATH, f"-Wl,-rpath,{lib_dir}"], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr
    n, bank, st, nb, fb, bad = map(int, run.stdout.split())
    assert n == len(syms) and bank == 16 and nb == 1 and fb == 1
    assert bad == _lib.STG_ERR_INVALID
    expect = (_lib.STG_OK,) if have_gpu() else (_lib.STG_ERR_NO_DEVICE,)
    assert st in expect
