"""Loaders for the oracle libraries (test infrastructure only).

* ``RefCpu``  oracle/_ref/libref_cpu.so  - the reference's own classes built with g++ (ref_harness.cpp)
* ``RefGpu``  oracle/_ref/libref_gpu.so  - the reference's own classes built with nvcc (ref_gpu_harness.cu)
* ``Port``    oracle/librt_port.so       - the CPU restatement in C (rt_port.c)

Each is None when its library has not been built (the reference-based ones need the reference tree
at build time; the built files then travel with the repository).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from cortexraytracercuda_b200.scene import RenderParams, Scene, SceneDesc, SceneFile

ORACLE = Path(__file__).resolve().parent.parent / "oracle"
# the reference tree (flarive/CortexRaytracerCuda), used only to build the reference-based checkers:
# RTC_REFERENCE, else a checkout named `reference` beside this repository
REFERENCE = Path(os.environ.get("RTC_REFERENCE", str(ORACLE.parent.parent / "reference")))


def _load(path: Path):
    if not path.exists():
        return None
    return C.CDLL(str(path))


class _Base:
    prefix = ""

    def __init__(self, lib):
        self.lib = lib
        f = getattr(lib, self.prefix + "scene_create")
        f.restype = C.c_void_p
        getattr(lib, self.prefix + "last_error").restype = C.c_char_p
        getattr(lib, self.prefix + "scene_destroy").argtypes = [C.c_void_p]

    def error(self) -> str:
        return getattr(self.lib, self.prefix + "last_error")().decode()


class RefCpu(_Base):
    prefix = "refh_"

    def scene(self, scene: Scene, bvh_kind: int = -1):
        d = scene if isinstance(scene, SceneFile) else SceneDesc(scene)
        h = self.lib.refh_scene_create(d.ptr(), C.c_int(bvh_kind))
        if not h:
            raise RuntimeError(self.error())
        return _RefCpuScene(self, h, d)

    def rng_draws(self, seed: int, n: int) -> np.ndarray:
        out = np.empty(n, np.float32)
        self.lib.refh_rng_draws(C.c_uint32(seed), C.c_int64(n), out.ctypes.data_as(C.c_void_p))
        return out

    def get_int(self, seed: int, lo: int, hi: int, n: int) -> np.ndarray:
        out = np.empty(n, np.int32)
        self.lib.refh_get_int(C.c_uint32(seed), C.c_int(lo), C.c_int(hi), C.c_int64(n), out.ctypes.data_as(C.c_void_p))
        return out

    def sampler_draws(self, which: int, seed: int, n: int) -> np.ndarray:
        out = np.empty((n, 3), np.float32)
        rc = self.lib.refh_sampler_draws(C.c_int(which), C.c_uint32(seed), C.c_int64(n), out.ctypes.data_as(C.c_void_p))
        assert rc == 0
        return out


class _RefCpuScene:
    def __init__(self, o: RefCpu, h, d):
        self.o, self.h, self.d = o, C.c_void_p(h), d

    def __del__(self):
        try:
            self.o.lib.refh_scene_destroy(self.h)
        except Exception:
            pass

    def render_pixels(self, params: RenderParams, pix: np.ndarray, threads: int = 0):
        pix = np.ascontiguousarray(pix, dtype=np.int64)
        out = np.empty((pix.size, 4), np.float32)
        rays = C.c_uint64(0)
        p = params.to_c()
        rc = self.o.lib.refh_render_pixels(self.h, C.byref(p), pix.ctypes.data_as(C.c_void_p), C.c_int64(pix.size),
                                           out.ctypes.data_as(C.c_void_p), C.byref(rays), C.c_int(threads))
        if rc:
            raise RuntimeError(self.o.error())
        return out, rays.value

    def trace_closest(self, rays: np.ndarray, depth: int, max_depth: int):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        prim = np.empty(rays.shape[0], np.int32)
        t = np.empty(rays.shape[0], np.float32)
        rc = self.o.lib.refh_trace_closest(self.h, rays.ctypes.data_as(C.c_void_p), C.c_int64(rays.shape[0]),
                                           C.c_int(depth), C.c_int(max_depth), prim.ctypes.data_as(C.c_void_p),
                                           t.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError(self.o.error())
        return prim, t

    def camera_rays(self, params: RenderParams, i: int, j: int) -> np.ndarray:
        q = int(np.sqrt(np.float64(params.spp)))
        out = np.empty((q * q, 7), np.float32)
        p = params.to_c()
        self.o.lib.refh_camera_rays(self.h, C.byref(p), C.c_int(i), C.c_int(j), out.ctypes.data_as(C.c_void_p))
        return out


class RefGpu(_Base):
    prefix = "refg_"

    def __init__(self, lib):
        super().__init__(lib)
        self._setup = False

    def setup(self):
        if not self._setup:
            if self.lib.refg_setup() != 0:
                raise RuntimeError(self.error())
            self._setup = True

    def scene(self, scene: Scene):
        self.setup()
        d = scene if isinstance(scene, SceneFile) else SceneDesc(scene)
        h = self.lib.refg_scene_create(d.ptr())
        if not h:
            raise RuntimeError(self.error())
        return _RefGpuScene(self, h, d)

    def sampler_draws(self, which: int, seed: int, n: int) -> np.ndarray:
        self.setup()
        out = np.empty((n, 3), np.float32)
        rc = self.lib.refg_sampler_draws(C.c_int(which), C.c_uint32(seed), C.c_int64(n), out.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError(self.error())
        return out


class _RefGpuScene:
    def __init__(self, o: RefGpu, h, d):
        self.o, self.h, self.d = o, C.c_void_p(h), d

    def __del__(self):
        try:
            self.o.lib.refg_scene_destroy(self.h)
        except Exception:
            pass

    def render_pixels(self, params: RenderParams, pix: np.ndarray):
        pix = np.ascontiguousarray(pix, dtype=np.int64)
        out = np.empty((pix.size, 4), np.float32)
        p = params.to_c()
        rc = self.o.lib.refg_render_pixels(self.h, C.byref(p), pix.ctypes.data_as(C.c_void_p), C.c_int64(pix.size),
                                           out.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError(self.o.error())
        return out

    def render_frame_timed(self, params: RenderParams, want_image: bool = False):
        """The whole frame in the reference's launch shape (16x16 blocks, one thread per pixel); returns
        (kernel milliseconds from CUDA events, (H, W, 4) sums or None)."""
        ms = C.c_float(0.0)
        img = np.empty((params.height, params.width, 4), np.float32) if want_image else None
        p = params.to_c()
        rc = self.o.lib.refg_render_frame_timed(self.h, C.byref(p), img.ctypes.data_as(C.c_void_p) if want_image else None,
                                                C.byref(ms))
        if rc:
            raise RuntimeError(self.o.error())
        return float(ms.value), img

    def trace_closest(self, rays: np.ndarray, depth: int, max_depth: int):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        prim = np.empty(rays.shape[0], np.int32)
        t = np.empty(rays.shape[0], np.float32)
        rc = self.o.lib.refg_trace_closest(self.h, rays.ctypes.data_as(C.c_void_p), C.c_int64(rays.shape[0]),
                                           C.c_int(depth), C.c_int(max_depth), prim.ctypes.data_as(C.c_void_p),
                                           t.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError(self.o.error())
        return prim, t


class Port:
    """The C restatement (oracle/rt_port.c).  trig=0: glibc float cos/sin/acos/atan2 (bit-exact with
    the reference's g++ build); trig=1: double-evaluated and rounded (bit-exact with the compat kernel)."""

    def __init__(self, lib):
        self.lib = lib
        lib.port_scene_create.restype = C.c_void_p
        lib.port_scene_destroy.argtypes = [C.c_void_p]
        lib.port_last_error.restype = C.c_char_p

    def set_trig(self, mode: int):
        self.lib.port_set_trig(C.c_int(mode))

    def scene(self, scene: Scene):
        d = scene if isinstance(scene, SceneFile) else SceneDesc(scene)
        h = self.lib.port_scene_create(d.ptr())
        if not h:
            raise RuntimeError(self.lib.port_last_error().decode())
        return _PortScene(self, h, d)

    def sphere_light_draws(self, seed: int, n: int) -> np.ndarray:
        """omni_light::random for the known-answer light (see port_sphere_light_draws)."""
        out = np.empty((n, 3), np.float32)
        self.lib.port_sphere_light_draws(C.c_uint32(seed), C.c_int64(n), out.ctypes.data_as(C.c_void_p))
        return out

    def rng_draws(self, seed: int, n: int) -> np.ndarray:
        out = np.empty(n, np.float32)
        self.lib.port_rng_draws(C.c_uint32(seed), C.c_int64(n), out.ctypes.data_as(C.c_void_p))
        return out


class _PortScene:
    def __init__(self, o: Port, h, d):
        self.o, self.h, self.d = o, C.c_void_p(h), d

    def __del__(self):
        try:
            self.o.lib.port_scene_destroy(self.h)
        except Exception:
            pass

    def render_pixels(self, params: RenderParams, pix: np.ndarray, threads: int = 8, trig: int = 0):
        self.o.set_trig(trig)
        pix = np.ascontiguousarray(pix, dtype=np.int64)
        out = np.empty((pix.size, 4), np.float32)
        rays = C.c_uint64(0)
        p = params.to_c()
        rc = self.o.lib.port_render_pixels(self.h, C.byref(p), pix.ctypes.data_as(C.c_void_p), C.c_int64(pix.size),
                                           out.ctypes.data_as(C.c_void_p), C.byref(rays), C.c_int(threads))
        self.o.set_trig(0)
        if rc:
            raise RuntimeError(self.o.lib.port_last_error().decode())
        return out, rays.value

    def trace_closest(self, rays: np.ndarray, depth: int, max_depth: int):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        prim = np.empty(rays.shape[0], np.int32)
        t = np.empty(rays.shape[0], np.float32)
        self.o.lib.port_trace_closest(self.h, rays.ctypes.data_as(C.c_void_p), C.c_int64(rays.shape[0]), C.c_int(depth),
                                      C.c_int(max_depth), prim.ctypes.data_as(C.c_void_p), t.ctypes.data_as(C.c_void_p))
        return prim, t


def port():
    lib = _load(ORACLE / "librt_port.so")
    return Port(lib) if lib else None


class Fp64:
    """The double-precision clean-mode estimator (oracle/fp64_clean.c): converged-image reference."""

    def __init__(self, lib):
        self.lib = lib
        lib.f64_scene_create.restype = C.c_void_p
        lib.f64_scene_destroy.argtypes = [C.c_void_p]
        lib.f64_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_void_p,
                                   C.c_int64, C.c_void_p, C.c_int]

    def set_bvh_threshold(self, min_prims: int):
        """Scenes created afterwards search closest hits through a tree above `min_prims` primitives."""
        self.lib.f64_set_bvh_threshold(C.c_int(min_prims))

    def render(self, scene: Scene, width: int, height: int, spp: int, max_depth: int, seed: int,
               pix: np.ndarray | None = None, threads: int = 0) -> np.ndarray:
        """Radiance sums (n, 3) float64 of the given frame-buffer pixels (all pixels by default)."""
        import os
        d = scene if isinstance(scene, SceneFile) else SceneDesc(scene)
        h = self.lib.f64_scene_create(d.ptr())
        try:
            if pix is None:
                pix = np.arange(width * height, dtype=np.int64)
            pix = np.ascontiguousarray(pix, dtype=np.int64)
            out = np.empty((pix.size, 3), np.float64)
            self.lib.f64_render(h, width, height, spp, max_depth, seed & 0xFFFFFFFF, pix.ctypes.data, pix.size,
                                out.ctypes.data, threads or (os.cpu_count() or 1))
        finally:
            self.lib.f64_scene_destroy(h)
        return out


def fp64():
    lib = _load(ORACLE / "librt_fp64.so")
    return Fp64(lib) if lib else None


def ref_cpu():
    lib = _load(ORACLE / "_ref" / "libref_cpu.so")
    return RefCpu(lib) if lib else None


def ref_gpu():
    lib = _load(ORACLE / "_ref" / "libref_gpu.so")
    return RefGpu(lib) if lib else None


# ------------------------------------------------------------------------------------------------
# parity metrics
# ------------------------------------------------------------------------------------------------
def parity_stats(ours: np.ndarray, ref: np.ndarray, rel_tol: float = 1e-4):
    """Per-pixel comparison of RGB sums.  A pixel matches when every channel satisfies
    |a - b| <= rel_tol * max(|b|, floor) with floor = 1e-3 * mean(|ref|) (dark pixels)."""
    a = np.asarray(ours, np.float64)[..., :3].reshape(-1, 3)
    b = np.asarray(ref, np.float64)[..., :3].reshape(-1, 3)
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    nan_mismatch = int(np.any(nan_a != nan_b, axis=1).sum())
    a0 = np.where(nan_a, 0.0, a)
    b0 = np.where(nan_b, 0.0, b)
    floor = 1e-3 * max(float(np.abs(b0).mean()), 1e-12)
    err = np.abs(a0 - b0) / np.maximum(np.abs(b0), floor)
    pix_err = err.max(axis=1)
    ok = pix_err <= rel_tol
    rmse = float(np.sqrt(((a0 - b0) ** 2).mean()) / max(float(np.sqrt((b0 ** 2).mean())), 1e-12))
    exact = float(np.all(a0 == b0, axis=1).mean())
    mean_rel = float(abs(a0.mean() - b0.mean()) / max(abs(b0.mean()), 1e-12))
    return {"frac_ok": float(ok.mean()), "frac_exact": exact, "rel_rmse": rmse, "mean_rel": mean_rel,
            "max_pix_err": float(pix_err.max()), "nan_mismatch": nan_mismatch, "n": int(a.shape[0])}


# ------------------------------------------------------------------------------------------------
# thrust::minstd_rand in Python (small n) and the reference's multi-draw helpers in both orders
# ------------------------------------------------------------------------------------------------
M31 = 2147483647


def minstd_uniform(seed: int, n: int) -> np.ndarray:
    x = seed % M31
    if x == 0:
        x = 1
    out = np.empty(n, np.float32)
    for k in range(n):
        x = (x * 48271) % M31
        out[k] = np.float32(x - 1) * np.float32(2.0 ** -31)
    return out


def sampler_reproduction(which: int, seed: int, n: int, order: int) -> np.ndarray:
    """random_in_unit_disk (0), random_in_unit_sphere (1), random_cosine_direction (2) and
    directional_light::random for P=0, u=x, v=y from o=0 (3); order 0 = left to right."""
    f = np.float32
    u = minstd_uniform(seed, 8 * n + 64)
    k = 0
    res = []

    def take(m):
        nonlocal k
        vals = [u[k + i] for i in range(m)]
        k += m
        return vals if order == 0 else vals[::-1]

    while len(res) < n:
        if which == 0:
            a, b = take(2)
            px, py = f(2) * a - f(1), f(2) * b - f(1)
            if f(f(px * px) + f(py * py)) + f(0) < f(1):
                res.append((px, py, 0.0))
        elif which == 1:
            a, b, c = take(3)
            px, py, pz = f(2) * a - f(1), f(2) * b - f(1), f(2) * c - f(1)
            if f(f(f(px * px) + f(py * py)) + f(pz * pz)) < f(1):
                res.append((px, py, pz))
        elif which == 2:
            r1, r2 = u[k], u[k + 1]
            k += 2
            phi = f(6.28318530718) * r1
            z = np.sqrt(f(1) - r2)
            s = np.sqrt(r2)
            res.append((f(np.cos(np.float64(phi))) * s, f(np.sin(np.float64(phi))) * s, z))
        else:
            a, b = take(2)
            res.append((a - f(0.5), b - f(0.5), 0.0))
    return np.array(res, np.float32)
