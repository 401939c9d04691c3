"""Python host API over the C ABI, mirroring the reference's renderer interface.

Reference interface (flarive/CortexRaytracerCuda):
  * ``class renderer { virtual void render(const sceneConfig&, const render_parameters&) const = 0; }``
    (core/src/renderers/renderer.h:16), implemented for CUDA by ``gpu_cuda_renderer``
    (core/src/renderers/gpu_cuda_renderer.h:23-27), which calls
  * ``launchGPU(sceneCfg, width, height, spp, max_depth, tx=16, ty=16, filepath, quiet=true)``
    (core/src/gpu.cu:2127).

Here ``GpuB200Renderer.render(scene, params)`` renders a :class:`~.scene.Scene` with
:class:`RenderParameters` (the CLI-level ``render_parameters`` of misc/render_parameters.h:13-103:
width, height, spp, max depth, save path, quiet) and ``launch_gpu`` has launchGPU's arguments.
Errors raise :class:`RtcError` (the reference prints and exits(99), gpu.cu:119-129).
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import RtcError, check
from .scene import (MODE_COMPAT, DRAW_ORDER_DEVICE, REQ_DONE, REQ_FAILED, Camera, RenderParams, Scene, SceneDesc,
                    rtc_batch_params, rtc_job, rtc_render_stats, rtc_request, rtc_request_info, rtc_scene_info, rtc_scene_options,
                    rtc_server_config, rtc_server_stats)


def _desc(scene):
    """A Scene's packed description, or a SceneFile as it is (both have .ptr())."""
    return scene if hasattr(scene, "ptr") and not isinstance(scene, Scene) else SceneDesc(scene)


class Context:
    """One CUDA device + stream (rtc_context)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.rtc_context_create(device, C.byref(h)))
        self.handle = h
        self._scenes = weakref.WeakSet()

    def close(self):
        if self.handle:
            for s in list(self._scenes):
                s.close()
            self.lib.rtc_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, scene: Scene) -> "DeviceScene":
        return DeviceScene(self, scene)

    def render_batch(self, jobs, slots: int = 0, ring: int = 0, batch: int = 0, drain: int = 0,
                     stream: int | None = None, d_counters: int | None = None, block: int = 0) -> None:
        """Renders many images through one wavefront (rtc_render_batch).  ``jobs`` are :class:`Job`s whose
        ``d_radiance`` device buffers receive each image's radiance sums; returns when all are complete."""
        arr = (rtc_job * max(1, len(jobs)))()
        cams = []
        for k, j in enumerate(jobs):
            cam = None
            if j.camera is not None:
                c = j.camera.to_c()
                cams.append(c)
                cam = C.pointer(c)
            arr[k] = rtc_job(j.scene.handle.value, cam, j.params.to_c(), j.d_radiance)
        bp = rtc_batch_params(slots, ring, batch, drain, d_counters, block)
        check(self.lib.rtc_render_batch(self.handle, arr, len(jobs), C.byref(bp),
                                        C.c_void_p(stream) if stream else None))

    def last_stats(self) -> dict:
        """Statistics of the last render (iterations, launches, drained slots, bulk/drain device ms)."""
        st = rtc_render_stats()
        check(self.lib.rtc_get_render_stats(self.handle, C.byref(st)))
        return {k: getattr(st, k) for k, _ in rtc_render_stats._fields_}


class DeviceScene:
    """A flattened scene resident on the device (rtc_scene): BVH, primitives, textures.  `bvh_builder`:
    BVH_SAH (host binned SAH, default), BVH_DEVICE (PLOC built on the device) or BVH_DEVICE_LBVH (linear
    BVH built on the device)."""

    def __init__(self, ctx: Context, scene: Scene, bvh_builder: int = 0):
        self.ctx = ctx
        self.desc = _desc(scene)
        h = C.c_void_p()
        if not ctx.handle:
            raise RtcError(1, "context is closed")
        opt = rtc_scene_options(bvh_builder)
        check(ctx.lib.rtc_scene_create_ex(ctx.handle, self.desc.ptr(), C.byref(opt), C.byref(h)))
        self.handle = h
        ctx._scenes.add(self)

    def info(self) -> dict:
        i = rtc_scene_info()
        check(self.ctx.lib.rtc_scene_get_info(self.handle, C.byref(i)))
        return {k: getattr(i, k) for k, _ in rtc_scene_info._fields_}

    def close(self):
        if self.handle:
            self.ctx.lib.rtc_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, params: RenderParams, want_rgb8: bool = False):
        """Renders into host buffers.  Returns (radiance_sum (H, W, 4) float32 in frame-buffer order,
        rgb8 (H, W, 3) uint8 in PNG order or None)."""
        n = params.width * params.height
        rad = np.empty((params.height, params.width, 4), np.float32)
        rgb = np.empty((params.height, params.width, 3), np.uint8) if want_rgb8 else None
        p = params.to_c()
        check(self.ctx.lib.rtc_render(self.ctx.handle, self.handle, C.byref(p), rad.ctypes.data,
                                      rgb.ctypes.data if rgb is not None else None))
        assert rad.size == 4 * n
        return rad, rgb

    def render_device(self, params: RenderParams, d_radiance: int, d_rgb8: int | None = None,
                      d_counters: int | None = None, stream: int | None = None):
        """Asynchronous render into device buffers (raw device pointers, e.g. torch tensor .data_ptr())."""
        p = params.to_c()
        check(self.ctx.lib.rtc_render_device(self.ctx.handle, self.handle, C.byref(p), C.c_void_p(d_radiance),
                                             C.c_void_p(d_rgb8) if d_rgb8 else None,
                                             C.c_void_p(d_counters) if d_counters else None,
                                             C.c_void_p(stream) if stream else None))

    def trace_closest(self, rays: np.ndarray, depth: int = 0, max_depth: int = 1, flags: int = 0):
        """Closest-hit primitive id (-1 = miss) and t for rays (n, 8) = (ox,oy,oz,tmin,dx,dy,dz,tmax).
        ``flags``: FLAG_WIDE_BVH walks the 8-wide nodes."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        check(self.ctx.lib.rtc_trace_closest_ex(self.ctx.handle, self.handle, rays.ctypes.data, n, depth, max_depth,
                                                flags, prim.ctypes.data, t.ctypes.data))
        return prim, t


@dataclass
class Job:
    """One image of a batched render: a resident scene, its parameters, a device output buffer
    (width*height float4, e.g. a torch tensor's data_ptr()) and optionally its own camera."""
    scene: DeviceScene
    params: RenderParams
    d_radiance: int
    camera: Camera | None = None


def _host_ptr(buf) -> int:
    if hasattr(buf, "data_ptr"):
        return buf.data_ptr()
    return buf.ctypes.data


class RenderServer:
    """A render server on one device (rtc_server): requests are submitted while others render, admitted
    into the running wavefront as memory and ring entries free up, and copied to the caller's buffer
    when complete.  Scenes are registered once and kept resident under an HBM budget (LRU eviction)."""

    def __init__(self, device: int = 0, mode: int = MODE_COMPAT, draw_order: int = DRAW_ORDER_DEVICE,
                 slots: int = 0, ring: int = 0, batch: int = 0, hbm_budget_bytes: int = 0, flags: int = 0,
                 bvh_builder: int = 0):
        self.lib = _lib.load()
        cfg = rtc_server_config(device, mode, draw_order, batch, slots, ring, hbm_budget_bytes, flags, bvh_builder)
        h = C.c_void_p()
        check(self.lib.rtc_server_create(C.byref(cfg), C.byref(h)))
        self.handle = h
        self._outs = {}

    def close(self):
        if self.handle:
            self.lib.rtc_server_destroy(self.handle)
            self.handle = None
            self._outs.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, scene: Scene) -> int:
        desc = _desc(scene)
        sid = C.c_uint32()
        check(self.lib.rtc_server_add_scene(self.handle, desc.ptr(), C.byref(sid)))
        return sid.value

    def submit(self, scene_id: int, params: RenderParams, camera: Camera | None = None, out=None):
        """Queues a request; ``out`` (default: a new numpy array) is an (H, W, 4) float32 host buffer that
        receives the radiance sums.  Returns (ticket, out)."""
        if out is None:
            out = np.empty((params.height, params.width, 4), np.float32)
        req = rtc_request(scene_id, 1 if camera is None else 0, (camera or Camera()).to_c(), params.width,
                          params.height, params.spp, params.max_depth, params.seed & 0xFFFFFFFF)
        t = C.c_uint64()
        check(self.lib.rtc_server_submit(self.handle, C.byref(req), C.c_void_p(_host_ptr(out)), C.byref(t)))
        self._outs[t.value] = out
        return t.value, out

    @staticmethod
    def _info(i: rtc_request_info) -> dict:
        return {k: getattr(i, k) for k, _ in rtc_request_info._fields_}

    def poll(self, ticket: int):
        """(done, info): done once the result is in the buffer (the request is then released)."""
        i = rtc_request_info()
        r = self.lib.rtc_server_poll(self.handle, ticket, C.byref(i))
        if r == 10:   # RTC_ERR_BUSY
            return False, self._info(i)
        self._outs.pop(ticket, None)
        check(r)
        return True, self._info(i)

    def wait(self, ticket: int, timeout_ms: int = -1):
        """Blocks until the request is done; returns (out, info)."""
        i = rtc_request_info()
        r = self.lib.rtc_server_wait(self.handle, ticket, timeout_ms, C.byref(i))
        out = self._outs.pop(ticket, None) if r != 5 else self._outs.get(ticket)
        check(r)
        return out, self._info(i)

    def stats(self) -> dict:
        st = rtc_server_stats()
        check(self.lib.rtc_server_get_stats(self.handle, C.byref(st)))
        return {k: getattr(st, k) for k, _ in rtc_server_stats._fields_}


@dataclass
class RenderParameters:
    """The reference's render_parameters subset that reaches launchGPU (misc/render_parameters.h)."""
    width: int = 256
    height: int = 144          # 256 / (16/9), render_parameters.h:13-15
    spp: int = 100
    max_depth: int = 100
    save_filepath: str = "image.png"
    quiet: bool = True
    mode: int = MODE_COMPAT
    draw_order: int = DRAW_ORDER_DEVICE


class GpuB200Renderer:
    """Drop-in for gpu_cuda_renderer: render(scene, params) writes the PNG like launchGPU does."""

    def __init__(self, device: int = 0):
        self.ctx = Context(device)

    def render(self, scene: Scene, params: RenderParameters):
        ds = DeviceScene(self.ctx, scene)
        try:
            rp = RenderParams(params.width, params.height, params.spp, params.max_depth, 2580, params.mode,
                              params.draw_order)
            rad, rgb = ds.render(rp, want_rgb8=True)
            check(self.ctx.lib.rtc_write_png(params.save_filepath.encode(), rgb.ctypes.data, params.width,
                                             params.height))
            return rad, rgb
        finally:
            ds.close()


def launch_gpu(scene: Scene, width: int, height: int, spp: int, max_depth: int, tx: int = 16, ty: int = 16,
               filepath: str = "image.png", quiet: bool = True) -> None:
    """launchGPU (core/src/gpu.cu:2127) through the C ABI's rtc_launchGPU."""
    lib = _lib.load()
    d = SceneDesc(scene)
    check(lib.rtc_launchGPU(d.ptr(), width, height, spp, max_depth, tx, ty, filepath.encode(), int(bool(quiet))))


__all__ = ["Context", "DeviceScene", "GpuB200Renderer", "RenderParameters", "launch_gpu", "RtcError"]
