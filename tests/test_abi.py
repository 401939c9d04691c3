"""The C-ABI library loads and exports every function include/rtc.h declares; host-only entry points
behave (argument checks, PNG writer, no-device status).  No kernel launches: CPU only."""
import ctypes as C
import re
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

from cortexraytracercuda_b200 import _lib, configs
from cortexraytracercuda_b200.scene import SceneDesc, rtc_render_params

HEADER = Path(__file__).resolve().parent.parent / "include" / "rtc.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rtc_[a-zA-Z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from cortexraytracercuda_b200.build import build
    build()
    return _lib.load()


def test_header_declares_expected_api():
    names = declared_functions()
    for n in ("rtc_context_create", "rtc_scene_create", "rtc_render", "rtc_render_device", "rtc_launchGPU",
              "rtc_trace_closest", "rtc_last_error_string", "rtc_write_png"):
        assert n in names


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the binding declares prototypes for all of them
    assert set(declared_functions()) <= set(_lib.PROTOTYPES)


def test_noalloc_cap_matches_header():
    m = re.search(r"#define\s+RTC_NOALLOC_MAX_PIXELS\s+(\d+)u?", HEADER.read_text())
    assert m and int(m.group(1)) == _lib.NOALLOC_MAX_PIXELS


def test_struct_sizes_match_header(lib):
    # the ctypes mirror and the C layout agree on the sizes the ABI depends on
    assert C.sizeof(rtc_render_params) == 10 * 4


def test_null_arguments_are_rejected(lib):
    out = C.c_void_p()
    assert lib.rtc_context_create(0, None) == 1
    assert lib.rtc_scene_create(None, None, C.byref(out)) == 1
    assert lib.rtc_render(None, None, None, None, None) == 1
    assert lib.rtc_scene_destroy(None) == 0
    assert lib.rtc_context_destroy(None) == 0
    assert b"null" in lib.rtc_last_error_string()


def test_no_device_status_without_gpu(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert lib.rtc_context_create(0, C.byref(h)) == 6   # RTC_ERR_NO_DEVICE, never exit()
    d = SceneDesc(configs.cornell())
    assert lib.rtc_launchGPU(d.ptr(), 8, 8, 1, 2, 16, 16, b"/tmp/never_written.png", 1) == 6


def test_png_writer_roundtrip(lib, tmp_path):
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, size=(17, 23, 3), dtype=np.uint8)
    path = tmp_path / "x.png"
    assert lib.rtc_write_png(str(path).encode(), img.ctypes.data, 23, 17) == 0
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert zlib.crc32(typ + body) & 0xffffffff == crc
        if typ == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
            assert (w, h) == (23, 17)
        if typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(17, 1 + 23 * 3)
    assert np.all(rows[:, 0] == 0)
    assert np.array_equal(rows[:, 1:].reshape(17, 23, 3), img)


def test_png_writer_bad_path(lib):
    img = np.zeros((2, 2, 3), np.uint8)
    assert lib.rtc_write_png(b"/nonexistent_dir/x.png", img.ctypes.data, 2, 2) == 7   # RTC_ERR_IO
