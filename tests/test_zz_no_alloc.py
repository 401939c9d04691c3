"""rtc_render_noalloc: the render entry point for callers that cannot allocate device memory when they
render (a memory budget fixed at start-up, a device allocator owned by another framework, a render
issued where a cudaMalloc would synchronise the device).  It must give the same image as the regular
device entry point, call after call, from its static scratch array.

This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from cortexraytracercuda_b200 import _lib, configs
from cortexraytracercuda_b200._lib import check
from cortexraytracercuda_b200.renderer import Context, DeviceScene
from cortexraytracercuda_b200.scene import DRAW_ORDER_DEVICE, MODE_COMPAT

import oracles

pytestmark = pytest.mark.gpu


def _noalloc(lib, ds, params, out):
    p = params.to_c()
    return lib.rtc_render_noalloc(ds.handle, C.byref(p), C.c_void_p(out.data_ptr()), None)


def test_noalloc_matches_render_device_on_consecutive_calls():
    import torch
    lib = _lib.load()
    with Context(0) as ctx:
        scene = configs.cornell()
        params = configs.cornell_params(width=200, height=150, spp=16, max_depth=8)
        params.mode, params.draw_order = MODE_COMPAT, DRAW_ORDER_DEVICE
        ds = DeviceScene(ctx, scene)
        ref = torch.empty((params.height, params.width, 4), dtype=torch.float32, device="cuda")
        ds.render_device(params, ref.data_ptr())
        torch.cuda.synchronize()
        ref_np = ref.cpu().numpy()
        small = params.__class__(**{**params.__dict__, "width": 37, "height": 23})
        for k in range(2):
            out = torch.full((params.height, params.width, 4), -1.0, dtype=torch.float32, device="cuda")
            check(_noalloc(lib, ds, params, out))
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            st = oracles.parity_stats(got.reshape(-1, 4), ref_np.reshape(-1, 4))
            assert st["frac_ok"] >= 0.99 and st["mean_rel"] <= 0.02, st   # the parity tolerance of the suite
            assert np.array_equal(got, ref_np)                             # same kernels: identical sums
            # a differently sized call in between must not leak state into the next call
            tmp = torch.empty((small.height, small.width, 4), dtype=torch.float32, device="cuda")
            check(_noalloc(lib, ds, small, tmp))
        ds.close()


def test_noalloc_rejects_images_beyond_its_scratch():
    import torch
    lib = _lib.load()
    with Context(0) as ctx:
        ds = DeviceScene(ctx, configs.cornell())
        side = int(np.ceil(np.sqrt(_lib.NOALLOC_MAX_PIXELS + 1)))
        params = configs.cornell_params(width=side, height=side, spp=1, max_depth=2)
        out = torch.empty(4, dtype=torch.float32, device="cuda")   # never written: rejected first
        rc = _noalloc(lib, ds, params, out)
        assert rc == 1   # RTC_ERR_INVALID_ARGUMENT
        assert b"at most" in lib.rtc_last_error_string()
        ds.close()
