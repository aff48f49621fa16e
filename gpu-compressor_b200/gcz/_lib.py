"""ctypes declarations of libgcz (include/gcz.h, include/gcz_gen.h).

The library is built in-tree (gpu-compressor_b200/build.py).  There is no
fallback: if libgcz.so is missing or does not load, importing gcz fails.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgcz.so")

GCZ_OK = 0
GCZ_EINVAL = -1
GCZ_ECUDA = -2
GCZ_ENOMEM = -3
GCZ_ECAPACITY = -4
GCZ_EDEVICE = -5
GCZ_ETOOLARGE = -6
GCZ_EUNAVAILABLE = -7
GCZ_ECODEC = -8
GCZ_ETIMEOUT = -9
NOALLOC_MAX_INPUT = 8 << 20

WINDOW = 65536
ZSTD_MAX_SEQ_PER_WINDOW = 21845
LZMA2_MAX_MATCHES = 8
LZMA2_SEARCH_DEPTH = 32

# Every symbol include/gcz.h and include/gcz_gen.h declare: name -> (restype, argtypes)
_vp, _cp = ctypes.c_void_p, ctypes.c_char_p
_i, _u32, _u64, _sz, _l, _d = ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_long, ctypes.c_double
SIGNATURES = {
    "gcz_create": (_i, [_i, ctypes.POINTER(_vp)]),
    "gcz_destroy": (None, [_vp]),
    "gcz_last_error": (_cp, [_vp]),
    "gcz_device": (_i, [_vp]),
    "gcz_version": (_cp, []),
    "gcz_set_option": (_i, [_vp, _cp, _l]),
    "gcz_sync": (_i, [_vp, _vp]),
    "gcz_query": (_i, [_vp, _cp, ctypes.POINTER(_l)]),
    "gcz_zstd_search_depth_for_level": (_u32, [_u32]),
    "gcz_num_windows": (_sz, [_sz]),
    "gcz_zstd_max_sequences": (_sz, [_sz]),
    "gcz_zstd_match_find": (_i, [_vp, _vp, _sz, _u32, _vp, _sz, _vp]),
    "gcz_zstd_match_find_packed": (_i, [_vp, _vp, _sz, _u32, _vp, _sz, _vp]),
    "gcz_zstd_match_find_device": (_i, [_vp, _vp, _sz, _u32, _vp, _sz, _vp, _vp]),
    "gcz_zstd_match_find_device_noalloc": (_i, [_i, _vp, _sz, _u32, _vp, _sz, _vp, _vp]),
    "gcz_zstd_match_find_ref_layout_device": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _u32, _u32, _u32, _u32, _u32, _vp]),
    "gcz_lzma2_match_find": (_i, [_vp, _vp, _sz, _u32, _vp, _vp]),
    "gcz_lzma2_match_find_device": (_i, [_vp, _vp, _sz, _u32, _vp, _vp, _vp]),
    "gcz_lzma2_find_matches": (_i, [_vp, _vp, _sz, _u32, _vp, _vp, _vp]),
    "gcz_lzma2_match_find_ref_layout_device": (_i, [_vp, _vp, _vp, _vp, _u32, _u32, _u32, _u32, _u32, _vp]),
    "gcz_batch_num_windows": (_sz, [_vp, _sz]),
    "gcz_batch_layout": (_i, [_vp, _sz, _vp, _vp, ctypes.POINTER(_u64)]),
    "gcz_zstd_match_find_batch_device": (_i, [_vp, _vp, _u64, _vp, _u32, _u32, _vp, _sz, _vp, _vp]),
    "gcz_lzma2_match_find_batch_device": (_i, [_vp, _vp, _u64, _vp, _u32, _u32, _vp, _vp, _vp]),
    "gcz_zstd_match_find_files": (_i, [_vp, _vp, _vp, _sz, _u32, _vp, _sz, _vp]),
    "gcz_server_create": (_i, [_vp, _u64, _u64, _u32, ctypes.POINTER(_vp)]),
    "gcz_server_destroy": (None, [_vp]),
    "gcz_server_max_batch_bytes": (_u64, [_vp]),
    "gcz_server_info": (_i, [_vp, ctypes.POINTER(_u32), ctypes.POINTER(_u64)]),
    "gcz_server_selftest_wait_timeout": (_i, [_vp, _u32, ctypes.POINTER(_u64)]),
    "gcz_server_submit": (_i, [_vp, _i, _u32, _vp, _sz, _vp, _sz, _vp, ctypes.POINTER(_u64)]),
    "gcz_server_wait": (_i, [_vp, _u64, _d, ctypes.POINTER(_d)]),
    "gcz_server_stats": (_i, [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                              ctypes.POINTER(_d), ctypes.POINTER(_d)]),
    "gcz_zstd_frames_bound": (_sz, [_sz]),
    "gcz_zstd_compress_frames": (_i, [_vp, _vp, _sz, _u32, _u32, _vp, _sz, _vp, ctypes.POINTER(_sz)]),
    "gcz_zstd_compress_frames_gpu": (_i, [_vp, _vp, _sz, _u32, _vp, _sz, _vp, ctypes.POINTER(_sz)]),
    "gcz_zstd_encode_frames_device": (_i, [_vp, _vp, _sz, _vp, _vp, _vp, _sz, _vp, _vp]),
    "gcz_selftest_wait_timeout": (_i, [_vp, _u32]),
    "gcz_zstd_encode_frames_batch_device": (_i, [_vp, _vp, _u64, _vp, _u32, _vp, _vp, _vp, _sz, _vp, _vp]),
    "gcz_zstd_compress_files_gpu": (_i, [_vp, _vp, _vp, _sz, _u32, _vp, _sz, _vp, ctypes.POINTER(_sz)]),
    "gcz_profile_start": (_i, [_vp]),
    "gcz_profile_stop": (_i, [_vp, ctypes.POINTER(_d), ctypes.POINTER(_u64), ctypes.POINTER(_u64)]),
    "gcz_gen_synthetic": (None, [_u64, _vp, _u64, _u64, _d, _d, _d]),
    "gcz_gen_file_sizes": (None, [_u64, _u64, _u64, _u64, _vp, _vp]),
}

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgcz.so not built ({LIB_PATH}); run gpu-compressor_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
