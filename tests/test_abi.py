"""CPU checks of the C-ABI boundary: the library loads without a GPU and
exports every function include/sph_b200.h declares; the Python struct layout
matches the C header."""
import ctypes
import os
import re
import subprocess

import pytest

import sph_b200 as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sph_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_]+\**\s+\**(sph_[a-z_]+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def built_lib():
    import build_lib as pkg_build
    pkg_build.build()
    return ctypes.CDLL(S.LIB_PATH)


def test_header_declares_expected_entry_points():
    fns = declared_functions()
    assert set(S.EXPORTED_SYMBOLS) == set(fns), fns


def test_library_exports_every_declared_symbol(built_lib):
    for name in declared_functions():
        assert hasattr(built_lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", S.LIB_PATH], capture_output=True, text=True).stdout
    for name in declared_functions():
        assert re.search(r"\bT\s+%s\b" % name, out), name


def test_strerror_without_device(built_lib):
    built_lib.sph_strerror.restype = ctypes.c_char_p
    assert built_lib.sph_strerror(0) == b"ok"
    assert b"capacity" in built_lib.sph_strerror(-2)
    assert built_lib.sph_strerror(-999) == b"unknown status"


def test_init_without_device_fails_cleanly(built_lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("device present")
    except Exception:
        pass
    lib = S.load()
    cfg = S.tgv_baseline_config(16)
    h = ctypes.c_void_p()
    assert lib.sph_init(ctypes.byref(cfg), 256, ctypes.byref(h)) == -10   # SPH_E_NODEVICE


def test_struct_sizes_match_header(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text('#include "sph_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                    'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(sph_config), sizeof(sph_diag),'
                    ' sizeof(sph_timings), offsetof(sph_config, cell_skin), sizeof(sph_adj_config),'
                    ' offsetof(sph_adj_config, target_vel), offsetof(sph_adj_config, body_motion));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals == [ctypes.sizeof(S.SphConfig), ctypes.sizeof(S.SphDiag), ctypes.sizeof(S.SphTimings),
                    S.SphConfig.cell_skin.offset, ctypes.sizeof(S.SphAdjConfig), S.SphAdjConfig.target_vel.offset,
                    S.SphAdjConfig.body_motion.offset]


def test_config_validation_codes():
    """Invalid configurations are rejected before any device work (sph_init
    checks the device first, so this exercises the Python-side presets)."""
    c = S.tgv_baseline_config(64)
    assert c.kernel_model == S.KERNEL_WENDLAND2 and c.kernel_scale == 2.0
    assert abs(c.h - 1.3 / 64) < 1e-15
    assert abs(S.baseline_dt(c) - 0.25 * c.h / 10.0) < 1e-18
    r = S.tgv_reference_config(100)
    assert r.kernel_model == S.KERNEL_GAUSSIAN and r.kernel_scale == 3.0 and r.rho0 == 1000.0


def test_restart_image_size(built_lib):
    """sph_restart_size: a 64-byte header and 108 bytes per particle (pos, vel 16
    each; rho, mass, smass 8 each; type, itype, label 4 each; carried drho 8,
    acc and avg 16 each); no device needed."""
    lib = S.load()
    assert lib.sph_restart_size(0) == 0
    assert lib.sph_restart_size(1) == 64 + 108
    assert lib.sph_restart_size(1000) == 64 + 108 * 1000
