"""ctypes binding of librtc_b200.so (the C ABI declared in include/rtc.h).

The library is built in-tree (``python -m cortexraytracercuda_b200.build``).  Loading fails loudly
when it is missing: there is no CPU fallback for the render path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .scene import (rtc_batch_params, rtc_job, rtc_obj_mesh, rtc_render_params, rtc_render_stats, rtc_request, rtc_request_info,
                    rtc_scene_desc, rtc_scene_info, rtc_scene_options, rtc_server_config, rtc_server_stats,
                    IMAGE_LOADER, rtc_scene_file_info)

LIB_PATH = Path(__file__).resolve().parent / "librtc_b200.so"

# include/rtc.h: RTC_NOALLOC_MAX_PIXELS
NOALLOC_MAX_PIXELS = 508376

STATUS_NAMES = {0: "RTC_OK", 1: "RTC_ERR_INVALID_ARGUMENT", 2: "RTC_ERR_BAD_SCENE", 3: "RTC_ERR_CUDA",
                4: "RTC_ERR_OOM", 5: "RTC_ERR_TIMEOUT", 6: "RTC_ERR_NO_DEVICE", 7: "RTC_ERR_IO",
                8: "RTC_ERR_DEVICE_CHECK", 9: "RTC_ERR_NOT_FOUND", 10: "RTC_ERR_BUSY"}

# every symbol include/rtc.h declares, with (restype, argtypes)
_P = C.c_void_p
PROTOTYPES = {
    "rtc_last_error_string": (C.c_char_p, []),
    "rtc_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "rtc_context_destroy": (C.c_int, [_P]),
    "rtc_scene_create": (C.c_int, [_P, C.POINTER(rtc_scene_desc), C.POINTER(C.c_void_p)]),
    "rtc_trace_closest_ex": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_int32, C.c_int32, C.c_int32, _P, _P]),
    "rtc_scene_create_ex": (C.c_int, [_P, C.POINTER(rtc_scene_desc), C.POINTER(rtc_scene_options),
                                      C.POINTER(C.c_void_p)]),
    "rtc_scene_destroy": (C.c_int, [_P]),
    "rtc_scene_get_info": (C.c_int, [_P, C.POINTER(rtc_scene_info)]),
    "rtc_render": (C.c_int, [_P, _P, C.POINTER(rtc_render_params), _P, _P]),
    "rtc_render_device": (C.c_int, [_P, _P, C.POINTER(rtc_render_params), _P, _P, _P, _P]),
    "rtc_render_noalloc": (C.c_int, [_P, C.POINTER(rtc_render_params), _P, _P]),
    "rtc_get_render_stats": (C.c_int, [_P, C.POINTER(rtc_render_stats)]),
    "rtc_render_batch": (C.c_int, [_P, C.POINTER(rtc_job), C.c_uint32, C.POINTER(rtc_batch_params), _P]),
    "rtc_server_create": (C.c_int, [C.POINTER(rtc_server_config), C.POINTER(C.c_void_p)]),
    "rtc_server_destroy": (C.c_int, [_P]),
    "rtc_server_add_scene": (C.c_int, [_P, C.POINTER(rtc_scene_desc), C.POINTER(C.c_uint32)]),
    "rtc_server_submit": (C.c_int, [_P, C.POINTER(rtc_request), _P, C.POINTER(C.c_uint64)]),
    "rtc_server_poll": (C.c_int, [_P, C.c_uint64, C.POINTER(rtc_request_info)]),
    "rtc_server_wait": (C.c_int, [_P, C.c_uint64, C.c_int32, C.POINTER(rtc_request_info)]),
    "rtc_server_get_stats": (C.c_int, [_P, C.POINTER(rtc_server_stats)]),
    "rtc_trace_closest": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_int32, C.c_int32, _P, _P]),
    "rtc_launchGPU": (C.c_int, [C.POINTER(rtc_scene_desc), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_char_p, C.c_int]),
    "rtc_load_obj": (C.c_int, [C.c_char_p, C.POINTER(rtc_obj_mesh)]),
    "rtc_scene_file_load": (C.c_int, [C.c_char_p, C.c_uint32, IMAGE_LOADER, C.c_void_p, C.POINTER(C.c_void_p)]),
    "rtc_scene_file_desc": (C.POINTER(rtc_scene_desc), [_P]),
    "rtc_scene_file_get_info": (C.c_int, [_P, C.POINTER(rtc_scene_file_info)]),
    "rtc_scene_file_skipped": (C.c_char_p, [_P, C.c_uint32]),
    "rtc_scene_file_free": (None, [_P]),
    "rtc_free_obj": (None, [C.POINTER(rtc_obj_mesh)]),
    "rtc_write_png": (C.c_int, [C.c_char_p, _P, C.c_int, C.c_int]),
}


class RtcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads the in-tree library (once) and declares the prototypes."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    # RTC_LIBRARY: load another build of the same ABI (variant builds of `build.py --out`)
    p = Path(path) if path else Path(os.environ.get("RTC_LIBRARY", LIB_PATH))
    if not p.exists():
        raise RtcError(-1, f"{p} is missing; build it with `python -m cortexraytracercuda_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int) -> None:
    if status != 0:
        msg = load().rtc_last_error_string()
        raise RtcError(status, msg.decode() if msg else "")
