"""The C-ABI library on a machine without a GPU: it loads, exports every symbol
the public headers declare (C names and the C++ names of the singlegemm entry
points), and its host-side argument checks behave like the reference's."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


@pytest.fixture(scope="module")
def fg():
    import flashgemm_b200 as fg
    from flashgemm_b200 import build
    build.build()
    fg.lib()
    return fg


def declared_symbols():
    names = set()
    for h in os.listdir(INC):
        text = open(os.path.join(INC, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:extern\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, re.M):
            if m.group(1) not in ("if", "while", "return", "defined"):
                names.add(m.group(1))
        for m in re.finditer(r"^extern\s+int\s+(\w+)\s*;", text, re.M):
            names.add(m.group(1))
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_every_declared_symbol_is_exported(fg):
    decl = declared_symbols()
    # the reference's public API (multigemm/src/flashgemm.h:17-25, singlegemm entry points)
    for must in ["flashgemm_thread_num", "flashgemm_set_thread_num", "flashgemm_multi_f32f32f32",
                 "flashgemm_multi_bf16bf16f32", "flashgemm_multi_int8uint8int32",
                 "LibShalom_sgemm_mp", "LibShalom_set_thread_nums", "Small_NGM_NN_SGEMM",
                 "Small_MGN_NN_SGEMM", "fg_chain_dev", "fg_sgemm_dev", "fg_last_error"]:
        assert must in decl, must
    exported = exported_symbols(fg.LIB_PATH)
    missing = sorted(decl - exported)
    assert not missing, missing


def test_cxx_linkage_names_are_exported(fg):
    exported = exported_symbols(fg.LIB_PATH)
    for mangled in ["_Z18LibShalom_sgemm_mpiiPfS_S_lll", "_Z25LibShalom_set_thread_numsi",
                    "_Z18Small_NGM_NN_SGEMMPfS_S_llliii", "_Z18Small_MGN_NN_SGEMMPfS_S_llliii"]:
        assert mangled in exported, mangled


def test_library_needs_no_libcuda_to_load(fg):
    out = subprocess.run(["ldd", fg.LIB_PATH], capture_output=True, text=True).stdout
    assert "libcuda.so" not in out


def test_thread_num_knob(fg):
    fg.flashgemm_set_thread_num(8)
    assert fg.flashgemm_thread_num() == 8
    fg.flashgemm_set_thread_num(1)
    assert fg.flashgemm_thread_num() == 1


def test_odd_k_rejected_before_any_device_work(fg, capfd):
    """flashgemm.c:13-22: K % 2 != 0 prints and returns, C untouched."""
    B = np.zeros((63, 32), np.float32)
    A = np.zeros((16, 63), np.float32)
    C = np.full((16, 32), 5.0, np.float32)
    fg.flashgemm_multi_f32f32f32(C, B, 32, 1, A, 16, 63)
    assert "K must be a multiple of 2" in capfd.readouterr().out
    assert fg.last_status() == fg.FG_ERR_INVALID
    assert (C == 5.0).all()


def test_shape_mismatch_rejected(fg):
    B = np.zeros((64, 32), np.uint8)
    A1 = np.zeros((16, 64), np.int8)
    A2 = np.zeros((16, 18), np.int8)
    C = np.zeros((16, 32), np.int32)
    fg.flashgemm_multi_int8uint8int32(C, B, 32, 2, A1, 16, 64, A2, 16, 18)
    assert fg.last_status() == fg.FG_ERR_INVALID
    assert "previous M" in fg.last_error()


def test_noalloc_arguments_checked_before_device_work(fg):
    """The allocation-free BF16 chain refuses bad shapes, strides and alignments on
    the host, before any CUDA call (the addresses below are never dereferenced)."""
    import ctypes
    L = fg.lib()
    f = L.fg_chain_bf16_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_long),
                  ctypes.POINTER(ctypes.c_long), ctypes.c_void_p, ctypes.c_void_p]

    def call(N, Ms, Ks, C=0x10000, B=0x20000, A=0x30000):
        n = len(Ms)
        As = (ctypes.c_void_p * n)(*[A + 0x1000 * i for i in range(n)])
        return f(C, B, N, n, As, (ctypes.c_long * n)(*Ms), (ctypes.c_long * n)(*Ks), None, None)

    cases = [
        (dict(N=(1 << 30) + 8, Ms=[64], Ks=[64]), "2^30"),
        (dict(N=100, Ms=[64], Ks=[64]), "multiple of 8"),
        (dict(N=256, Ms=[64, 32], Ks=[64, 48]), "previous M"),
        (dict(N=256, Ms=[64], Ks=[60]), "multiple of 8"),
        (dict(N=256, Ms=[0], Ks=[64]), "positive"),
        (dict(N=256, Ms=[64], Ks=[64], B=0x20008), "16-byte aligned"),
        (dict(N=256, Ms=[64], Ks=[64], A=0x30004), "16-byte aligned"),
    ]
    for kw, text in cases:
        assert call(**kw) == fg.FG_ERR_INVALID, kw
        assert text in fg.last_error(), (kw, fg.last_error())


def test_device_chain_arguments_checked_before_device_work(fg):
    """fg_chain_dev refuses unknown dtypes, bad chains, odd K and unaligned operands on
    the host, and returns at once for N == 0 (addresses never dereferenced)."""
    import ctypes
    L = fg.lib()

    def call(dt, N, Ms, Ks, C=0x10000, B=0x20000, A=0x30000):
        n = len(Ms)
        As = (ctypes.c_void_p * max(n, 1))(*[A + 0x1000 * i for i in range(n)])
        Mv = (ctypes.c_long * max(n, 1))(*Ms)
        Kv = (ctypes.c_long * max(n, 1))(*Ks)
        return L.fg_chain_dev(dt, C, B, N, n, ctypes.cast(As, ctypes.c_void_p),
                              ctypes.cast(Mv, ctypes.c_void_p), ctypes.cast(Kv, ctypes.c_void_p),
                              None)

    cases = [
        (dict(dt=7, N=256, Ms=[64], Ks=[64]), "dtype"),
        (dict(dt=fg.FG_DT_BF16, N=256, Ms=[], Ks=[]), "num_gemm"),
        (dict(dt=fg.FG_DT_INT8, N=256, Ms=[64, 32], Ks=[64, 48]), "previous M"),
        (dict(dt=fg.FG_DT_BF16, N=256, Ms=[64], Ks=[63]), "multiple of 2"),
        (dict(dt=fg.FG_DT_F32, N=(1 << 30) + 1, Ms=[64], Ks=[64]), "too large"),
        (dict(dt=fg.FG_DT_BF16, N=256, Ms=[64], Ks=[64], C=0x10004), "16-byte aligned"),
    ]
    for kw, text in cases:
        assert call(**kw) == fg.FG_ERR_INVALID, kw
        assert text in fg.last_error(), (kw, fg.last_error())
    assert call(fg.FG_DT_BF16, 0, [64], [64]) == fg.FG_OK


def test_settings_round_trip(fg):
    fg.set_semantics("math")
    assert fg.get_semantics() == fg.FG_SEM_MATH
    fg.set_semantics("ref")
    assert fg.get_semantics() == fg.FG_SEM_REF
    assert "sm_100a" in fg.version()
    for mode in ("off", "always", "auto"):
        fg.set_narrow(mode)
        assert fg.get_narrow() == mode
    fg.set_narrow(7)  # anything else: the measured default
    assert fg.get_narrow() == "auto"


def test_group_config_round_trip(fg):
    fg.set_group_config(fg.FG_GROUP_SINGLE_256, fg.FG_ORDER_LEVELS)
    assert fg.get_group_config() == (fg.FG_GROUP_SINGLE_256, fg.FG_ORDER_LEVELS)
    fg.set_group_config(7, 9)  # out of range: back to the autotuner's choice
    assert fg.get_group_config() == (fg.FG_GROUP_AUTO, fg.FG_ORDER_AUTO)


def test_autotune_table_file_round_trip(fg, tmp_path):
    """The remembered (kernel, order) choices survive a save / load; malformed
    lines and out-of-range choices are skipped. Host-only: no device needed."""
    src = tmp_path / "in.txt"
    sig_a = "0/0;256:1024x512,512x1024"
    sig_b = "1/0;64:64x64"
    src.write_text(f"0 1 {sig_a}\n2 0 {sig_b}\nnot a line\n5 0 3/0;1:1x1\n")
    fg.autotune_load(src)
    out = tmp_path / "out.txt"
    fg.autotune_save(out)
    lines = out.read_text().splitlines()
    assert f"0 1 {sig_a}" in lines and f"2 0 {sig_b}" in lines
    assert not any("3/0;1:1x1" in l for l in lines)
    with pytest.raises(fg.FlashgemmError):
        fg.autotune_load(tmp_path / "missing.txt")


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-device path")
def test_server_and_group_calls_report_no_device(fg):
    with pytest.raises(fg.FlashgemmError) as e:
        fg.Server()
    assert e.value.status == fg.FG_ERR_NO_DEVICE
    L = fg.lib()
    import ctypes
    L.fg_chain_group.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    assert L.fg_chain_group(fg.FG_DT_BF16, 0, None, None) != fg.FG_OK
