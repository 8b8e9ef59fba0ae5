"""The C-ABI library loads on a machine without a GPU and exports every entry point
declared in include/idx2g.h; host-only entry points work without a device."""
import ctypes
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "idx2g.h")).read()
    return sorted(set(re.findall(r"IDX2G_API\s+[\w\s\*]+?\b(idx2g_\w+)\s*\(", src)))


def test_all_declared_symbols_exported(idx2g):
    syms = declared_symbols()
    assert len(syms) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", idx2g.lib_path], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (idx2g_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    L = idx2g.lib()
    for s in syms:
        assert hasattr(L, s)


def test_params_defaults(idx2g):
    cp = idx2g._lib._CParams()
    idx2g.lib().idx2g_params_init(ctypes.byref(cp))
    assert list(cp.brick_dims) == [32, 32, 32]
    assert cp.bricks_per_chunk == 4096 and cp.chunks_per_file == 64 and cp.files_per_dir == 64
    assert cp.bit_planes_per_chunk == 1 and cp.bit_planes_per_file == 16
    assert list(cp.version) == [1, 0] and cp.out_dir == b"."


def test_version_string(idx2g):
    idx2g.lib().idx2g_version.restype = ctypes.c_char_p
    assert b"sm_100a" in idx2g.lib().idx2g_version()


def test_null_arguments_rejected(idx2g):
    L = idx2g.lib()
    assert L.idx2g_check_params(None) == 101
    assert L.idx2g_encode(None, None, None, 0, None) == 101
    assert L.idx2g_decode(None, None, None, None, 0, 0, None) == 101
