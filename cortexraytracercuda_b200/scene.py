"""Host-side scene description: a Python mirror of the C structs in include/rtc.h.

The reference describes a scene as a ``sceneConfig`` POD tree with uint8_t per-type counts, built by
``scene_builder`` from a libconfig ``.scene`` file (core/src/scenes/scene_config.h:452-459,
core/src/scenes/scene_builder.cpp).  Here a scene is built programmatically with the same object
vocabulary - textures, materials, directional lights, spheres, quads, triangle meshes, a perspective
camera and a background - and handed to the C ABI as one ``rtc_scene_desc``.

Objects keep the reference's load order (core/src/gpu.cu:504-635): directional lights, spheres, quads,
meshes.  The global primitive id of an object is its position in that order.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

# --- enums (rtc.h) -------------------------------------------------------------------------------
TEX_SOLID, TEX_CHECKER, TEX_IMAGE = 0, 1, 2
MAT_LAMBERTIAN, MAT_METAL, MAT_DIELECTRIC, MAT_DIFFUSE_LIGHT = 0, 1, 2, 3
BG_CONSTANT, BG_SKY_GRADIENT, BG_ENV_MAP = 0, 1, 2
MODE_COMPAT, MODE_CLEAN = 0, 1
ENGINE_AUTO, ENGINE_MEGAKERNEL, ENGINE_WAVEFRONT = 0, 1, 2
FLAG_KERNEL_TIMING = 1
FLAG_WIDE_BVH = 2
FLAG_SAMPLE_GROUPS = 4
FLAG_ENV_SAMPLING = 8   # clean mode: lambertian bounces also sample the environment map by luminance
BVH_SAH = 0        # binned SAH on host threads (default)
BVH_DEVICE = 1     # built on the device: Morton sort + PLOC clustering (near-SAH quality)
BVH_DEVICE_LBVH = 2   # built on the device: Morton sort + linear BVH (fastest build)
DRAW_ORDER_DEVICE, DRAW_ORDER_HOST = 0, 1

F3 = C.c_float * 3


class rtc_texture(C.Structure):
    _fields_ = [("kind", C.c_int32), ("color", F3), ("scale", C.c_float), ("even", C.c_int32),
                ("odd", C.c_int32), ("image", C.c_int32)]


class rtc_image(C.Structure):
    _fields_ = [("rgb", C.POINTER(C.c_uint8)), ("width", C.c_int32), ("height", C.c_int32)]


class rtc_material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("texture", C.c_int32), ("fuzz", C.c_float), ("ior", C.c_float),
                ("intensity", C.c_float), ("directional", C.c_int32)]


class rtc_sphere(C.Structure):
    _fields_ = [("center", F3), ("radius", C.c_float), ("material", C.c_int32)]


class rtc_quad(C.Structure):
    _fields_ = [("q", F3), ("u", F3), ("v", F3), ("material", C.c_int32)]


class rtc_dir_light(C.Structure):
    _fields_ = [("position", F3), ("u", F3), ("v", F3), ("color", F3), ("intensity", C.c_float),
                ("invisible", C.c_int32)]


class rtc_omni_light(C.Structure):
    _fields_ = [("position", F3), ("radius", C.c_float), ("color", F3), ("intensity", C.c_float),
                ("invisible", C.c_int32)]


class rtc_spot_light(C.Structure):
    _fields_ = [("position", F3), ("direction", F3), ("cutoff", C.c_float), ("falloff", C.c_float),
                ("intensity", C.c_float), ("radius", C.c_float), ("color", F3), ("invisible", C.c_int32)]


class rtc_mesh(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("indices", C.POINTER(C.c_uint32)),
                ("normals", C.POINTER(C.c_float)), ("uvs", C.POINTER(C.c_float)),
                ("num_vertices", C.c_uint32), ("num_triangles", C.c_uint32), ("material", C.c_int32),
                ("smooth", C.c_int32)]


class rtc_camera(C.Structure):
    _fields_ = [("look_from", F3), ("look_at", F3), ("up", F3), ("vfov", C.c_float), ("aspect", C.c_float),
                ("aperture", C.c_float), ("focus", C.c_float)]


class rtc_background(C.Structure):
    _fields_ = [("kind", C.c_int32), ("color", F3), ("top", F3), ("env_rgb", C.POINTER(C.c_float)),
                ("env_width", C.c_int32), ("env_height", C.c_int32)]


XF_TRANSLATE, XF_ROTATE, XF_SCALE = 1, 2, 4


class rtc_transform(C.Structure):
    _fields_ = [("translate", F3), ("rotate", F3), ("scale", F3), ("flags", C.c_uint32)]


class rtc_box(C.Structure):
    _fields_ = [("center", F3), ("size", F3), ("material", C.c_int32), ("transform", C.c_uint32)]


class rtc_scene_desc(C.Structure):
    _fields_ = [("textures", C.POINTER(rtc_texture)), ("num_textures", C.c_uint32),
                ("images", C.POINTER(rtc_image)), ("num_images", C.c_uint32),
                ("materials", C.POINTER(rtc_material)), ("num_materials", C.c_uint32),
                ("dir_lights", C.POINTER(rtc_dir_light)), ("num_dir_lights", C.c_uint32),
                ("spheres", C.POINTER(rtc_sphere)), ("num_spheres", C.c_uint32),
                ("quads", C.POINTER(rtc_quad)), ("num_quads", C.c_uint32),
                ("meshes", C.POINTER(rtc_mesh)), ("num_meshes", C.c_uint32),
                ("camera", rtc_camera), ("background", rtc_background),
                ("omni_lights", C.POINTER(rtc_omni_light)), ("num_omni_lights", C.c_uint32),
                ("spot_lights", C.POINTER(rtc_spot_light)), ("num_spot_lights", C.c_uint32),
                ("transforms", C.POINTER(rtc_transform)), ("num_transforms", C.c_uint32),
                ("sphere_transforms", C.POINTER(C.c_uint32)), ("quad_transforms", C.POINTER(C.c_uint32)),
                ("mesh_transforms", C.POINTER(C.c_uint32)),
                ("boxes", C.POINTER(rtc_box)), ("num_boxes", C.c_uint32)]


class rtc_render_params(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("seed", C.c_uint32), ("mode", C.c_int32), ("draw_order", C.c_int32),
                ("block_size", C.c_int32), ("engine", C.c_int32), ("flags", C.c_int32)]


class rtc_render_stats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("launches", C.c_uint32), ("drained_slots", C.c_uint32),
                ("engine", C.c_uint32), ("bulk_ms", C.c_float), ("drain_ms", C.c_float), ("extend_ms", C.c_float),
                ("shade_ms", C.c_float), ("extend_launches", C.c_uint32), ("shade_launches", C.c_uint32)]


class rtc_scene_info(C.Structure):
    _fields_ = [("num_primitives", C.c_uint32), ("num_lights", C.c_uint32), ("num_nodes", C.c_uint32),
                ("max_leaf_size", C.c_uint32), ("device_bytes", C.c_uint64), ("build_ms", C.c_double),
                ("bvh_builder", C.c_uint32), ("num_wide_nodes", C.c_uint32)]


class rtc_scene_options(C.Structure):
    _fields_ = [("bvh_builder", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class rtc_obj_mesh(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)), ("uvs", C.POINTER(C.c_float)),
                ("indices", C.POINTER(C.c_uint32)), ("num_vertices", C.c_uint32), ("num_triangles", C.c_uint32)]


class rtc_job(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", C.POINTER(rtc_camera)), ("params", rtc_render_params),
                ("d_radiance_sum", C.c_void_p)]


class rtc_batch_params(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("ring", C.c_uint32), ("batch", C.c_int32), ("drain", C.c_uint32),
                ("d_counters", C.c_void_p), ("block", C.c_uint32)]


class rtc_server_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("mode", C.c_int32), ("draw_order", C.c_int32), ("batch", C.c_int32),
                ("slots", C.c_uint32), ("ring", C.c_uint32), ("hbm_budget_bytes", C.c_uint64),
                ("flags", C.c_int32), ("bvh_builder", C.c_uint32)]


class rtc_request(C.Structure):
    _fields_ = [("scene_id", C.c_uint32), ("use_scene_camera", C.c_int32), ("camera", rtc_camera),
                ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("seed", C.c_uint32)]


class rtc_request_info(C.Structure):
    _fields_ = [("state", C.c_int32), ("scene_uploaded", C.c_int32), ("submit_ms", C.c_double),
                ("admit_ms", C.c_double), ("done_ms", C.c_double), ("paths", C.c_uint64)]


class rtc_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64), ("paths", C.c_uint64),
                ("scene_uploads", C.c_uint64), ("scene_evictions", C.c_uint64), ("resident_bytes", C.c_uint64),
                ("peak_resident_bytes", C.c_uint64), ("iterations", C.c_uint64), ("launches", C.c_uint64),
                ("queued", C.c_uint32), ("in_flight", C.c_uint32)]


REQ_QUEUED, REQ_RUNNING, REQ_COPYING, REQ_DONE, REQ_FAILED = range(5)


def _f3(v) -> F3:
    v = [float(x) for x in v]
    if len(v) != 3:
        raise ValueError("expected 3 components")
    return F3(*v)


def _carray(ctype, items):
    arr = (ctype * max(1, len(items)))()
    for k, it in enumerate(items):
        arr[k] = it
    return arr


def _carray_rows(ctype, kinds: str, rows):
    """A ctypes array of `ctype` (a structure of 4-byte fields, F3 counted as three) built in one pass
    from flat rows of numbers in field order: `kinds` has 'f' (float) or 'i' (int32) per word.  The
    same bytes as constructing each element, at numpy speed (the spheres frame's 489 spheres, materials
    and textures took 2 ms one ctypes element at a time)."""
    n = len(rows)
    words = len(kinds)
    assert C.sizeof(ctype) == 4 * words
    buf = np.zeros((max(1, n), words), np.uint32)
    if n:
        vals = np.asarray(rows, dtype=np.float64).reshape(n, words)
        for j, k in enumerate(kinds):
            col = vals[:, j]
            buf[:n, j] = col.astype(np.float32).view(np.uint32) if k == "f" else col.astype(np.int64).astype(np.int32).view(np.uint32)
    arr = (ctype * max(1, n)).from_buffer(buf)
    arr._rows = buf   # the array views this buffer: keep it alive with it
    return arr


def _texture_row(t):
    if t[0] == "solid":
        c = t[1]
        return (TEX_SOLID, c[0], c[1], c[2], 0.0, -1, -1, -1)
    if t[0] == "checker":
        return (TEX_CHECKER, 0.0, 0.0, 0.0, t[1], t[2], t[3], -1)
    return (TEX_IMAGE, 0.0, 0.0, 0.0, 0.0, -1, -1, t[1])


@dataclass
class Camera:
    look_from: tuple = (0.0, 0.0, 10.0)
    look_at: tuple = (0.0, 0.0, 0.0)
    up: tuple = (0.0, 1.0, 0.0)
    vfov: float = 70.0
    aspect: float = 16.0 / 9.0      # scene_builder's default camera (scene_builder.cpp:49)
    aperture: float = 0.0
    focus: float = 100.0

    def to_c(self) -> rtc_camera:
        return rtc_camera(_f3(self.look_from), _f3(self.look_at), _f3(self.up), self.vfov, self.aspect,
                          self.aperture, self.focus)


@dataclass
class RenderParams:
    width: int
    height: int
    spp: int
    max_depth: int
    seed: int = 2580               # core/src/gpu.cu:2080
    mode: int = MODE_COMPAT
    draw_order: int = DRAW_ORDER_DEVICE
    block_size: int = 0
    engine: int = ENGINE_AUTO
    flags: int = 0

    def to_c(self) -> rtc_render_params:
        return rtc_render_params(self.width, self.height, self.spp, self.max_depth, self.seed & 0xFFFFFFFF,
                                 self.mode, self.draw_order, self.block_size, self.engine, self.flags)

    @property
    def traced_spp(self) -> int:
        """Samples actually traced per pixel: int(sqrt(spp))^2 in compat mode (gpu.cu:1989)."""
        if self.mode == MODE_COMPAT:
            q = int(np.sqrt(np.float32(self.spp)))
            return q * q
        return self.spp


@dataclass
class Scene:
    """A scene under construction.  ``add_*`` return the index of what they add."""
    textures: list = field(default_factory=list)
    images: list = field(default_factory=list)        # (H, W, 3) uint8 arrays, top row first
    materials: list = field(default_factory=list)
    dir_lights: list = field(default_factory=list)
    omni_lights: list = field(default_factory=list)
    spot_lights: list = field(default_factory=list)
    spheres: list = field(default_factory=list)
    quads: list = field(default_factory=list)
    meshes: list = field(default_factory=list)        # dicts with numpy arrays
    boxes: list = field(default_factory=list)         # (center, size, material, transform ref)
    transforms: list = field(default_factory=list)    # (translate, rotate, scale, flags)
    sphere_transforms: dict = field(default_factory=dict)   # sphere index -> 1-based transform ref
    quad_transforms: dict = field(default_factory=dict)
    camera: Camera = field(default_factory=Camera)
    background: dict = field(default_factory=lambda: {"kind": BG_CONSTANT, "color": (0.0, 0.0, 0.0)})
    name: str = "scene"

    # textures -------------------------------------------------------------------------------------
    def solid(self, rgb) -> int:
        self.textures.append(("solid", tuple(float(x) for x in rgb)))
        return len(self.textures) - 1

    def checker(self, scale, even_tex: int, odd_tex: int) -> int:
        self.textures.append(("checker", float(scale), int(even_tex), int(odd_tex)))
        return len(self.textures) - 1

    def checker_colors(self, scale, odd_rgb, even_rgb) -> int:
        """scene_factory::createCheckerTexture(name, oddColor, evenColor, ..., scale) followed by
        checker_texture(scale, c1, c2): the odd colour lands in m_even and the even colour in m_odd
        (core/src/scene_factory.cuh:619-629 with checker_texture.cuh:28-31)."""
        return self.checker(scale, self.solid(odd_rgb), self.solid(even_rgb))

    def image(self, rgb: np.ndarray) -> int:
        rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
        if rgb.ndim != 3 or rgb.shape[2] != 3:
            raise ValueError("image must be (H, W, 3) uint8")
        self.images.append(rgb)
        img = len(self.images) - 1
        self.textures.append(("image", img))
        return len(self.textures) - 1

    # materials ------------------------------------------------------------------------------------
    def lambertian(self, tex_or_rgb) -> int:
        tex = tex_or_rgb if isinstance(tex_or_rgb, int) else self.solid(tex_or_rgb)
        self.materials.append((MAT_LAMBERTIAN, tex, 0.0, 0.0, 0.0, 0))
        return len(self.materials) - 1

    def metal(self, rgb, fuzz) -> int:
        tex = self.solid(rgb)
        f = float(fuzz)
        self.materials.append((MAT_METAL, tex, f if f < 1.0 else 1.0, 0.0, 0.0, 0))   # metal.cuh:52
        return len(self.materials) - 1

    def dielectric(self, ior) -> int:
        self.materials.append((MAT_DIELECTRIC, -1, 0.0, float(ior), 0.0, 0))
        return len(self.materials) - 1

    def diffuse_light(self, rgb, intensity=1.0, directional=True) -> int:
        tex = self.solid(rgb)
        self.materials.append((MAT_DIFFUSE_LIGHT, tex, 0.0, 0.0, float(intensity), int(bool(directional))))
        return len(self.materials) - 1

    # objects --------------------------------------------------------------------------------------
    def dir_light(self, position, u, v, rgb, intensity=1.0, invisible=True) -> int:
        self.dir_lights.append((tuple(position), tuple(u), tuple(v), tuple(rgb), float(intensity), int(bool(invisible))))
        return len(self.dir_lights) - 1

    def omni_light(self, position, radius, rgb, intensity=1.0, invisible=True) -> int:
        """An emitting sphere (omni_light); the light list puts omni lights first."""
        self.omni_lights.append((tuple(position), float(radius), tuple(rgb), float(intensity), int(bool(invisible))))
        return len(self.omni_lights) - 1

    def spot_light(self, position, direction, cutoff_deg, falloff, rgb, intensity=1.0, radius=0.1,
                   invisible=True) -> int:
        """An emitting sphere lit within `cutoff_deg` of `direction` (spot_light); listed after the
        directional lights."""
        self.spot_lights.append((tuple(position), tuple(direction), float(cutoff_deg), float(falloff), float(intensity),
                                 float(radius), tuple(rgb), int(bool(invisible))))
        return len(self.spot_lights) - 1

    def transform(self, translate=None, rotate=None, scale=None) -> int:
        """An rt::translate / rotate / scale chain (rotate in degrees about x, y, z); returns the 1-based
        reference that sphere(), quad(), box() and mesh() take as `transform` (0 = none)."""
        flags = (XF_TRANSLATE if translate is not None else 0) | (XF_ROTATE if rotate is not None else 0) | \
            (XF_SCALE if scale is not None else 0)
        self.transforms.append((tuple(translate or (0, 0, 0)), tuple(rotate or (0, 0, 0)), tuple(scale or (1, 1, 1)), flags))
        return len(self.transforms)

    def sphere(self, center, radius, mat, transform=0) -> int:
        self.spheres.append((tuple(center), float(radius), int(mat)))
        if transform:
            self.sphere_transforms[len(self.spheres) - 1] = int(transform)
        return len(self.spheres) - 1

    def quad(self, q, u, v, mat, transform=0) -> int:
        self.quads.append((tuple(q), tuple(u), tuple(v), int(mat)))
        if transform:
            self.quad_transforms[len(self.quads) - 1] = int(transform)
        return len(self.quads) - 1

    def box(self, center, size, mat, transform=0) -> int:
        """An axis-aligned box of six rectangles (box.cuh), after the quads in the object order."""
        self.boxes.append((tuple(center), tuple(size), int(mat), int(transform)))
        return len(self.boxes) - 1

    def mesh(self, vertices, indices, mat, normals=None, uvs=None, smooth=False, transform=0) -> int:
        m = {"vertices": np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3),
             "indices": np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3),
             "normals": None if normals is None else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3),
             "uvs": None if uvs is None else np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2),
             "material": int(mat), "smooth": int(bool(smooth)), "transform": int(transform)}
        self.meshes.append(m)
        return len(self.meshes) - 1

    # background -----------------------------------------------------------------------------------
    def set_background_constant(self, rgb):
        self.background = {"kind": BG_CONSTANT, "color": tuple(rgb)}

    def set_background_sky(self, bottom=(1.0, 1.0, 1.0), top=(0.5, 0.7, 1.0)):
        self.background = {"kind": BG_SKY_GRADIENT, "color": tuple(bottom), "top": tuple(top)}

    def set_background_env(self, env_rgb: np.ndarray):
        env = np.ascontiguousarray(env_rgb, dtype=np.float32)
        if env.ndim != 3 or env.shape[2] != 3:
            raise ValueError("env map must be (H, W, 3) float32")
        self.background = {"kind": BG_ENV_MAP, "env": env}

    # counts ---------------------------------------------------------------------------------------
    @property
    def num_triangles(self) -> int:
        return int(sum(m["indices"].shape[0] for m in self.meshes))

    @property
    def num_primitives(self) -> int:
        return len(self.dir_lights) + len(self.spheres) + len(self.quads) + 6 * len(self.boxes) + self.num_triangles

    # C description --------------------------------------------------------------------------------
    def to_desc(self) -> "SceneDesc":
        return SceneDesc(self)


class SceneDesc:
    """Owns the ctypes arrays behind one rtc_scene_desc; keep it alive while the desc is in use."""

    def __init__(self, s: Scene):
        keep = []
        for t in s.textures:
            if t[0] == "solid" and len(t[1]) != 3:
                raise ValueError("expected 3 components")
        for (c, _r, _m) in s.spheres:
            if len(c) != 3:
                raise ValueError("expected 3 components")
        texs = _carray_rows(rtc_texture, "iffffiii", [_texture_row(t) for t in s.textures])
        imgs = []
        for im in s.images:
            keep.append(im)
            imgs.append(rtc_image(im.ctypes.data_as(C.POINTER(C.c_uint8)), im.shape[1], im.shape[0]))
        mats = _carray_rows(rtc_material, "iifffi", s.materials)
        lights = [rtc_dir_light(_f3(p), _f3(u), _f3(v), _f3(c), i, inv) for (p, u, v, c, i, inv) in s.dir_lights]
        omnis = [rtc_omni_light(_f3(p), r, _f3(c), i, inv) for (p, r, c, i, inv) in s.omni_lights]
        spots = [rtc_spot_light(_f3(p), _f3(d), cu, fo, i, r, _f3(c), inv)
                 for (p, d, cu, fo, i, r, c, inv) in s.spot_lights]
        spheres = _carray_rows(rtc_sphere, "ffffi", [(c[0], c[1], c[2], r, m) for (c, r, m) in s.spheres])
        quads = [rtc_quad(_f3(q), _f3(u), _f3(v), m) for (q, u, v, m) in s.quads]
        meshes = []
        for m in s.meshes:
            keep.extend([m["vertices"], m["indices"]])
            nrm = None
            uv = None
            if m["normals"] is not None:
                keep.append(m["normals"])
                nrm = m["normals"].ctypes.data_as(C.POINTER(C.c_float))
            if m["uvs"] is not None:
                keep.append(m["uvs"])
                uv = m["uvs"].ctypes.data_as(C.POINTER(C.c_float))
            meshes.append(rtc_mesh(m["vertices"].ctypes.data_as(C.POINTER(C.c_float)),
                                   m["indices"].ctypes.data_as(C.POINTER(C.c_uint32)),
                                   nrm, uv, m["vertices"].shape[0], m["indices"].shape[0], m["material"], m["smooth"]))
        cam = s.camera
        bg = s.background
        env_ptr = None
        ew = eh = 0
        if bg["kind"] == BG_ENV_MAP:
            keep.append(bg["env"])
            env_ptr = bg["env"].ctypes.data_as(C.POINTER(C.c_float))
            eh, ew = bg["env"].shape[:2]
        cbg = rtc_background(bg["kind"], _f3(bg.get("color", (0, 0, 0))), _f3(bg.get("top", (0, 0, 0))), env_ptr, ew, eh)
        self.arrays = [texs, _carray(rtc_image, imgs), mats,
                       _carray(rtc_dir_light, lights), spheres, _carray(rtc_quad, quads),
                       _carray(rtc_mesh, meshes), _carray(rtc_omni_light, omnis), _carray(rtc_spot_light, spots)]
        a = self.arrays
        self.desc = rtc_scene_desc(a[0], len(s.textures), a[1], len(imgs), a[2], len(s.materials), a[3], len(lights),
                                   a[4], len(s.spheres), a[5], len(quads), a[6], len(meshes),
                                   rtc_camera(_f3(cam.look_from), _f3(cam.look_at), _f3(cam.up), cam.vfov, cam.aspect,
                                              cam.aperture, cam.focus), cbg, a[7], len(omnis), a[8], len(spots))
        xfs = [rtc_transform(_f3(t), _f3(r), _f3(sc), fl) for (t, r, sc, fl) in s.transforms]
        boxes = [rtc_box(_f3(c), _f3(sz), m, x) for (c, sz, m, x) in s.boxes]
        refs = {}
        for name, n, get in (("sphere", len(s.spheres), s.sphere_transforms.get),
                             ("quad", len(s.quads), s.quad_transforms.get),
                             ("mesh", len(s.meshes), lambda i: s.meshes[i].get("transform", 0))):
            r = [int(get(i) or 0) for i in range(n)]
            refs[name] = _carray(C.c_uint32, r) if any(r) else None
        self.arrays += [_carray(rtc_transform, xfs), _carray(rtc_box, boxes)]
        self.arrays += [r for r in refs.values() if r is not None]
        self.desc.transforms, self.desc.num_transforms = self.arrays[9], len(xfs)
        self.desc.boxes, self.desc.num_boxes = self.arrays[10], len(boxes)
        for name, r in refs.items():
            if r is not None:
                setattr(self.desc, name + "_transforms", C.cast(r, C.POINTER(C.c_uint32)))
        self._keep = keep
        self.scene = s

    def ptr(self):
        return C.byref(self.desc)


def load_obj(path):
    """Reads a Wavefront OBJ file through the library's reader (rtc_load_obj): returns (vertices (n, 3),
    indices (m, 3) uint32, normals (n, 3) or None, uvs (n, 2) or None) as numpy arrays, ready for
    Scene.mesh()."""
    from . import _lib
    lib = _lib.load()
    m = rtc_obj_mesh()
    _lib.check(lib.rtc_load_obj(str(path).encode(), C.byref(m)))
    try:
        nv, nt = m.num_vertices, m.num_triangles
        v = np.ctypeslib.as_array(m.vertices, shape=(nv, 3)).copy()
        f = np.ctypeslib.as_array(m.indices, shape=(nt, 3)).copy()
        n = np.ctypeslib.as_array(m.normals, shape=(nv, 3)).copy() if m.normals else None
        t = np.ctypeslib.as_array(m.uvs, shape=(nv, 2)).copy() if m.uvs else None
    finally:
        lib.rtc_free_obj(C.byref(m))
    return v, f, n, t


# ---- the reference's .scene files ------------------------------------------------------------------
SCENE_FILE_REFERENCE_CAPACITY = 1   # the reference's table capacities (list length mod 256; glass sized from `dielectric`)
SCENE_FILE_REFERENCE_MESHES = 2     # the reference's OBJ meshes (meshes[0]'s file for every entry, no position or transform)


class rtc_scene_file_info(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("num_skipped", C.c_uint32)]


IMAGE_LOADER = C.CFUNCTYPE(C.c_void_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p)


def decode_png(path) -> np.ndarray | None:
    """RGB8 pixels (H, W, 3) of an 8-bit non-interlaced PNG (greyscale, RGB, palette, with or without
    alpha; alpha dropped), or None for anything else."""
    import struct
    import zlib
    try:
        data = open(path, "rb").read()
    except OSError:
        return None
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        return None
    pos, idat, plte, hdr = 8, b"", None, None
    while pos + 8 <= len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"PLTE":
            plte = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    if hdr is None:
        return None
    w, h, depth, ctype, _, _, interlace = hdr
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}.get(ctype)
    if depth != 8 or interlace or ch is None:
        return None
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + w * ch)
    out = np.zeros((h, w * ch), np.int32)
    for y in range(h):   # PNG row filters (0 none, 1 sub, 2 up, 3 average, 4 Paeth)
        f, row = raw[y, 0], raw[y, 1:].astype(np.int32)
        prev = out[y - 1] if y else np.zeros(w * ch, np.int32)
        cur = np.zeros(w * ch, np.int32)
        for x in range(w * ch):
            a = cur[x - ch] if x >= ch else 0
            b = prev[x]
            c = prev[x - ch] if x >= ch else 0
            if f == 0:
                pr = 0
            elif f == 1:
                pr = a
            elif f == 2:
                pr = b
            elif f == 3:
                pr = (a + b) // 2
            else:
                p = a + b - c
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                pr = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[x] = (row[x] + pr) & 255
        out[y] = cur
    px = out.astype(np.uint8).reshape(h, w, ch)
    if ctype == 3:
        return plte[px[..., 0]] if plte is not None else None
    if ch in (1, 2):
        return np.repeat(px[..., :1], 3, axis=2)
    return np.ascontiguousarray(px[..., :3])


def _png_loader(path, w, h, user):
    px = decode_png(path.decode())
    if px is None:
        return None
    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    buf = libc.malloc(px.nbytes)
    if not buf:
        return None
    C.memmove(buf, px.ctypes.data, px.nbytes)
    w[0], h[0] = px.shape[1], px.shape[0]
    return buf


_PNG_LOADER = IMAGE_LOADER(_png_loader)


class SceneFile:
    """A reference `.scene` file read by the library (rtc_scene_file_load): usable wherever a Scene is
    (DeviceScene, RenderServer.add_scene).  Image textures are decoded with decode_png (PNG only)."""

    def __init__(self, path, flags: int = 0, decode_images: bool = True):
        from . import _lib
        self.lib = _lib.load()
        h = C.c_void_p()
        _lib.check(self.lib.rtc_scene_file_load(str(path).encode(), flags, _PNG_LOADER if decode_images else IMAGE_LOADER(),
                                                None, C.byref(h)))
        self.handle = h
        info = rtc_scene_file_info()
        _lib.check(self.lib.rtc_scene_file_get_info(h, C.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in rtc_scene_file_info._fields_}
        self.skipped = [self.lib.rtc_scene_file_skipped(h, i).decode() for i in range(info.num_skipped)]

    def ptr(self):
        return self.lib.rtc_scene_file_desc(self.handle)

    @property
    def desc(self) -> rtc_scene_desc:
        return self.ptr().contents

    def params(self, **kw) -> RenderParams:
        """RenderParams from the file's image section (width, height, samplesPerPixel, maxDepth)."""
        i = self.info
        base = {k: v for k, v in (("width", i["width"]), ("height", i["height"]), ("spp", i["spp"]),
                                  ("max_depth", i["max_depth"])) if v > 0}
        return RenderParams(**{**base, **kw})

    def close(self):
        if getattr(self, "handle", None):
            self.lib.rtc_scene_file_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
