"""The C-ABI library loads and exports every function include/*.h declares;
host-only helpers behave (no GPU needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = []
    for f in sorted(os.listdir(INCLUDE)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(gcz_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_headers_declare_entry_points():
    names = declared_functions()
    for must in ("gcz_create", "gcz_zstd_match_find", "gcz_zstd_match_find_device",
                 "gcz_zstd_match_find_ref_layout_device", "gcz_lzma2_match_find", "gcz_lzma2_find_matches",
                 "gcz_lzma2_match_find_ref_layout_device", "gcz_gen_synthetic"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import gcz._lib as lib

    L = lib.load()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # and the ctypes table covers every declaration
    assert set(declared_functions()) <= set(lib.SIGNATURES), set(declared_functions()) - set(lib.SIGNATURES)


def test_build_targets_sm100a_only():
    """The library is compiled for sm_100a and nothing else: the build recipe
    passes exactly one -gencode, arch=compute_100a,code=sm_100a.  (On a GPU,
    test_zstd_gpu checks the loaded image's architecture through gcz_query.)"""
    import build as gcz_build

    assert gcz_build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert not any("gencode" in f or "arch" in f for f in gcz_build.FLAGS)


def test_host_helpers():
    import gcz

    L = gcz.L
    assert gcz.num_windows(0) == 0
    assert gcz.num_windows(1) == 1
    assert gcz.num_windows(65536) == 1
    assert gcz.num_windows(65537) == 2
    # level -> search depth (compress_zstd_custom.rs:57-61)
    assert [gcz.search_depth_for_level(l) for l in (0, 1, 2, 3)] == [1, 16, 64, 1]
    assert L.gcz_zstd_max_sequences(0) == 0
    assert L.gcz_zstd_max_sequences(4) == 1
    assert L.gcz_zstd_max_sequences(65536) == 21845
    assert L.gcz_zstd_max_sequences(65536 * 3 + 7) == 3 * 21845 + 2
    assert gcz.L.gcz_version().startswith(b"gcz")


def test_create_rejects_bad_device_without_gpu():
    import gcz

    h = ctypes.c_void_p()
    assert gcz.L.gcz_create(-1, ctypes.byref(h)) == gcz._lib.GCZ_EINVAL
    assert gcz.L.gcz_create(4096, ctypes.byref(h)) == gcz._lib.GCZ_EINVAL


def test_null_context_is_an_error_not_a_crash():
    import gcz

    assert gcz.L.gcz_zstd_match_find(None, None, 0, 16, None, 0, None) == gcz._lib.GCZ_EINVAL
    assert gcz.L.gcz_lzma2_match_find(None, None, 0, 32, None, None) == gcz._lib.GCZ_EINVAL
    assert gcz.L.gcz_last_error(None) == b"null context"


def test_c_example_compiles_against_the_header(tmp_path):
    """The C host example builds with gcc against include/gcz.h and libgcz.so
    (no GPU needed to compile and link)."""
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "gpu-compressor_b200", "gcz")
    subprocess.run(["gcc", "-O2", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
                    os.path.join(root, "gpu-compressor_b200", "examples", "gcz_compress.c"),
                    "-L", libdir, "-lgcz", f"-Wl,-rpath,{libdir}", "-o", str(tmp_path / "gcz_compress")], check=True)
