"""Synthetic scenes for the measured workloads and the parity cases.

No public dataset is involved: every scene is generated from a seed (default 20261203).  The shapes,
sizes and value distributions follow the workloads the library is measured on:

* ``cornell``      - Cornell box: five 555-unit lambertian wall quads, a 130x105 ceiling quad light
                     (emission 15), two white boxes of 12 triangles each (165^3 rotated +15 deg about y,
                     165x330x165 rotated -18 deg), camera (278,278,-800) -> (278,278,0), vfov 40; 256^2,
                     16 spp, depth 8.  Wall and light placement follow data/scenes/cornell_box.scene.
* ``spheres``      - ground sphere r=1000, 22x22 grid of r=0.2 spheres at (a+0.9u, 0.2, b+0.9u'),
                     80% lambertian (albedo U^3*U^3) / 15% metal (U(0.5,1)^3, fuzz U(0,0.5)) / 5%
                     dielectric (1.5), three r=1 feature spheres; camera (13,2,3) -> 0, vfov 20,
                     aperture 0.1, focus 10; 1280x720, 64 spp, depth 50; sky-gradient background; the
                     quad light of data/scenes/random_spheres.scene so the lambertian mixture PDF has a
                     light to sample (with an empty light list the reference's mixture PDF returns NaN
                     for half the bounces, hittable_list.cuh:191-215).
* ``meshes``       - an icosphere subdivided to 327,680 triangles, radially displaced by 3-octave value
                     noise of amplitude 0.15, four instances (metal, dielectric, lambertian, lambertian
                     with an RGB8 image texture mapped through per-vertex texture coordinates) =
                     1,310,720 triangles; a checker ground quad with a 10-unit period; a
                     2048x1024 FP32 equirectangular environment map (sky gradient + Gaussian sun lobe);
                     1920x1080, 128 spp, depth 16; plus a hidden 8x4 quad light above the instances, for the
                     same reason as in ``spheres``.
* ``textured``     - spheres and quads with checker and image textures (parity of the texture paths).
* batched workload (:func:`batch_workload`) - 64 heterogeneous scenes drawn from the seed: triangle
                     counts log-uniform in [1K, 500K] (instances of one displaced icosphere level) plus
                     20-120 random r=0.2 spheres, the ``spheres`` material mix (80/15/5 %), a ground
                     sphere, a quad light and a sky; resolutions uniform over {256^2, 512^2, 768x432,
                     1024^2}, spp uniform over {4, 16, 64}, depth uniform in 8..32.  The served workload
                     draws requests over these scenes (Zipf popularity, orbiting cameras).
* ``icosphere``    - a 1,280-triangle icosphere with lambertian, metal and dielectric instances.
"""
from __future__ import annotations

import math

import numpy as np

from .scene import Camera, RenderParams, Scene

DEFAULT_SEED = 20261203


# -------------------------------------------------------------------------------------------------
# geometry helpers
# -------------------------------------------------------------------------------------------------
def box_mesh(size, center, yaw_deg):
    """12-triangle box of extent `size` centred at `center`, rotated by `yaw_deg` about +y."""
    sx, sy, sz = (0.5 * float(s) for s in size)
    corners = np.array([[x, y, z] for x in (-sx, sx) for y in (-sy, sy) for z in (-sz, sz)], dtype=np.float64)
    th = math.radians(yaw_deg)
    c, s = math.cos(th), math.sin(th)
    rot = np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
    verts = corners @ rot.T + np.asarray(center, dtype=np.float64)
    # corner index = 4*ix + 2*iy + iz
    faces = [
        (0, 1, 3), (0, 3, 2),   # x-
        (4, 6, 7), (4, 7, 5),   # x+
        (0, 4, 5), (0, 5, 1),   # y-
        (2, 3, 7), (2, 7, 6),   # y+
        (0, 2, 6), (0, 6, 4),   # z-
        (1, 5, 7), (1, 7, 3),   # z+
    ]
    return verts.astype(np.float32), np.array(faces, dtype=np.uint32)


def icosphere(level: int):
    """Unit icosphere by repeated 4:1 edge-midpoint subdivision (20*4^level faces)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mid], axis=0)
        nf = f.shape[0]
        a = inv[:nf] + base
        b = inv[nf:2 * nf] + base
        c = inv[2 * nf:] + base
        f = np.concatenate([np.stack([f[:, 0], a, c], 1), np.stack([f[:, 1], b, a], 1),
                            np.stack([f[:, 2], c, b], 1), np.stack([a, b, c], 1)], axis=0)
    return v, f.astype(np.uint32)


def _lattice_hash(ix, iy, iz, seed):
    h = (ix.astype(np.int64) * 73856093) ^ (iy.astype(np.int64) * 19349663) ^ (iz.astype(np.int64) * 83492791) ^ seed
    h = (h ^ (h >> 13)) * 1274126177
    h = h ^ (h >> 16)
    return (h & 0xFFFFFF).astype(np.float64) / float(0xFFFFFF)


def value_noise(p: np.ndarray, octaves=3, base_freq=2.0, seed=DEFAULT_SEED):
    """Sum of `octaves` octaves of trilinear lattice value noise in [-1, 1] (amplitude halving)."""
    out = np.zeros(p.shape[0])
    amp, freq, norm = 1.0, base_freq, 0.0
    for o in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        fr = q - i0
        w = fr * fr * (3.0 - 2.0 * fr)
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    val = _lattice_hash(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed + 7919 * o)
                    wx = w[:, 0] if dx else 1.0 - w[:, 0]
                    wy = w[:, 1] if dy else 1.0 - w[:, 1]
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    acc += wx * wy * wz * val
        out += amp * (2.0 * acc - 1.0)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return out / norm


def displaced_icosphere(level: int, amplitude=0.15, seed=DEFAULT_SEED):
    v, f = icosphere(level)
    r = 1.0 + amplitude * value_noise(v, seed=seed)
    return (v * r[:, None]), f


def sphere_uvs(vertices) -> np.ndarray:
    """Per-vertex texture coordinates of a mesh around the origin: longitude and latitude of each vertex's
    direction (u = 0.5 + atan2(z, x) / 2pi, v = 0.5 + asin(y) / pi), as float32 (n, 2)."""
    d = np.asarray(vertices, np.float64)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    u = 0.5 + np.arctan2(d[:, 2], d[:, 0]) / (2.0 * math.pi)
    v = 0.5 + np.arcsin(np.clip(d[:, 1], -1.0, 1.0)) / math.pi
    return np.stack([u, v], axis=1).astype(np.float32)


def procedural_image(w: int, h: int, seed=DEFAULT_SEED):
    """Seeded RGB8 test image: smooth colour ramps plus a coarse random tile pattern."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    tiles = rng.integers(0, 256, size=(8, 8, 3))
    t = tiles[(y * 8) // h, (x * 8) // w]
    img = np.stack([(x * 255) // max(1, w - 1), (y * 255) // max(1, h - 1), (x ^ y) & 255], axis=-1)
    return ((img + t) // 2).astype(np.uint8)


def sky_sun_envmap(w=2048, h=1024, sun_dir=(0.35, 0.6, -0.72), sun_sigma=0.04, sun_power=40.0):
    """FP32 equirect map: sky gradient + Gaussian sun lobe, indexed as get_spherical_uv maps
    directions (u = (atan2(-z, x) + pi) / 2pi, v = acos(-y) / pi; row 0 = v near 1, i.e. up)."""
    j, i = np.mgrid[0:h, 0:w]
    u = (i + 0.5) / w
    v = 1.0 - (j + 0.5) / h
    phi = u * 2.0 * np.pi - np.pi
    theta = v * np.pi
    dy = -np.cos(theta)
    st = np.sin(theta)
    dx = np.cos(phi) * st
    dz = -np.sin(phi) * st
    a = 0.5 * (dy + 1.0)
    sky = (1.0 - a)[..., None] * np.array([1.0, 1.0, 1.0]) + a[..., None] * np.array([0.5, 0.7, 1.0])
    sd = np.asarray(sun_dir, dtype=np.float64)
    sd /= np.linalg.norm(sd)
    cosang = np.clip(dx * sd[0] + dy * sd[1] + dz * sd[2], -1.0, 1.0)
    ang = np.arccos(cosang)
    sun = sun_power * np.exp(-0.5 * (ang / sun_sigma) ** 2)
    env = sky + sun[..., None] * np.array([1.0, 0.95, 0.85])
    return env.astype(np.float32)


# -------------------------------------------------------------------------------------------------
# scenes
# -------------------------------------------------------------------------------------------------
def cornell(light_intensity=1.0) -> Scene:
    s = Scene(name="cornell")
    red = s.lambertian((0.65, 0.05, 0.05))
    green = s.lambertian((0.12, 0.45, 0.15))
    white = s.lambertian((0.73, 0.73, 0.73))
    s.dir_light((278.0, 554.0, 332.0), (-130.0, 0.0, 0.0), (0.0, 0.0, -105.0), (15.0, 15.0, 15.0),
                intensity=light_intensity, invisible=True)
    s.quad((555, 0, 0), (0, 555, 0), (0, 0, 555), green)
    s.quad((0, 0, 0), (0, 555, 0), (0, 0, 555), red)
    s.quad((0, 0, 0), (555, 0, 0), (0, 0, 555), white)
    s.quad((555, 555, 555), (-555, 0, 0), (0, 0, -555), white)
    s.quad((0, 0, 555), (555, 0, 0), (0, 555, 0), white)
    v1, f1 = box_mesh((165, 165, 165), (212.5, 82.5, 147.5), 15.0)
    v2, f2 = box_mesh((165, 330, 165), (347.5, 165.0, 377.5), -18.0)
    s.mesh(v1, f1, white)
    s.mesh(v2, f2, white)
    s.camera = Camera(look_from=(278, 278, -800), look_at=(278, 278, 0), up=(0, 1, 0), vfov=40.0, aspect=1.0,
                      aperture=0.0, focus=100.0)
    s.set_background_constant((0.0, 0.0, 0.0))
    return s


def _rot_inv(deg):
    """rt::rotate's inverse matrix (rotations by -x, -y, -z degrees about x, then y, then z), in double."""
    m = np.eye(3)
    for ax, a in enumerate(deg):
        c, s_ = np.cos(np.radians(-a)), np.sin(np.radians(-a))
        r = np.eye(3)
        i, j = [(1, 2), (0, 2), (0, 1)][ax]
        r[i, i], r[j, j] = c, c
        r[i, j], r[j, i] = (-s_, s_) if ax != 1 else (s_, -s_)
        m = m @ r
    return m


def placed(s: Scene, at, rotate=None, scale=None) -> int:
    """A transform that puts the object's origin at world point `at`.  The reference applies translate
    inside rotate and scale (world = s * R(p + t)), so t = R_inv(at / s)."""
    sc = np.ones(3) if scale is None else np.asarray(scale, float)
    t = np.asarray(at, float) / sc
    if rotate is not None:
        t = _rot_inv(rotate) @ t
    return s.transform(translate=tuple(float(x) for x in t), rotate=rotate, scale=scale)


def transforms_scene(seed=DEFAULT_SEED, multi_axis=True) -> Scene:
    """The Cornell room with the reference's own box primitives under transforms (the two boxes of
    cornell_box.scene, turned about y), a scaled glass sphere, a turned metal quad and an untransformed
    box; with `multi_axis`, also a box and a small displaced icosphere turned about two and three axes
    and scaled.  The reference culls a multi-axis rotation by corners mapped with its forward matrix,
    which is not where its inverse-mapped rays find the object, so those two objects differ at their
    edges from the reference's own build; the kernel and the C restatement agree on them."""
    s = Scene(name="xforms")
    red = s.lambertian((0.65, 0.05, 0.05))
    green = s.lambertian((0.12, 0.45, 0.15))
    white = s.lambertian((0.73, 0.73, 0.73))
    blue = s.lambertian((0.2, 0.3, 0.75))
    s.dir_light((278.0, 554.0, 332.0), (-130.0, 0.0, 0.0), (0.0, 0.0, -105.0), (15.0, 15.0, 15.0),
                intensity=1.0, invisible=True)
    s.quad((555, 0, 0), (0, 555, 0), (0, 0, 555), green)
    s.quad((0, 0, 0), (0, 555, 0), (0, 0, 555), red)
    s.quad((0, 0, 0), (555, 0, 0), (0, 0, 555), white)
    s.quad((555, 555, 555), (-555, 0, 0), (0, 0, -555), white)
    s.quad((0, 0, 555), (555, 0, 0), (0, 555, 0), white)
    s.quad((-60, -60, 0), (120, 0, 0), (0, 120, 0), s.metal((0.85, 0.85, 0.9), 0.05),
           transform=placed(s, (450, 300, 520), rotate=(0.0, 25.0, 0.0)))
    s.sphere((0, 0, 0), 1.0, s.dielectric(1.5), transform=placed(s, (150, 380, 250), scale=(60, 45, 60)))
    s.box((0, 0, 0), (165, 330, 165), white, transform=placed(s, (347.5, 165.0, 377.5), rotate=(0, -15, 0)))
    s.box((0, 0, 0), (165, 165, 165), white, transform=placed(s, (212.5, 82.5, 147.5), rotate=(0, 18, 0)))
    s.box((90, 470, 470), (60, 60, 60), red)
    if multi_axis:
        s.box((0, 0, 0), (70, 70, 70), blue, transform=placed(s, (440, 60, 110), rotate=(30, 40, 0), scale=(1.0, 1.2, 1.0)))
        v, f = displaced_icosphere(2, 0.1, seed)
        s.mesh(v, f, s.metal((0.9, 0.8, 0.5), 0.2),
               transform=placed(s, (300, 430, 200), rotate=(20, 35, 10), scale=(55, 55, 55)))
    s.camera = Camera(look_from=(278, 278, -800), look_at=(278, 278, 0), up=(0, 1, 0), vfov=40.0, aspect=1.0,
                      aperture=0.0, focus=100.0)
    s.set_background_constant((0.0, 0.0, 0.0))
    return s


def transforms_params(**kw) -> RenderParams:
    p = dict(width=64, height=64, spp=16, max_depth=8)
    p.update(kw)
    return RenderParams(**p)


def cornell_params(**kw) -> RenderParams:
    p = dict(width=256, height=256, spp=16, max_depth=8)
    p.update(kw)
    return RenderParams(**p)


def spheres(seed=DEFAULT_SEED, grid=11, light=True, sky=True) -> Scene:
    rng = np.random.default_rng(seed)
    s = Scene(name="spheres")
    if light:
        # data/scenes/random_spheres.scene:31-45
        s.dir_light((0.0, 554.0, 147.0), (300.0, 0.0, 0.0), (0.0, 0.0, 265.0), (7.0, 7.0, 7.0), intensity=1.5,
                    invisible=True)
    ground = s.lambertian((0.5, 0.5, 0.5))
    s.sphere((0.0, -1000.0, 0.0), 1000.0, ground)
    s.sphere((0.0, 1.0, 0.0), 1.0, s.dielectric(1.5))
    s.sphere((-4.0, 1.0, 0.0), 1.0, s.lambertian((0.4, 0.2, 0.1)))
    s.sphere((4.0, 1.0, 0.0), 1.0, s.metal((0.7, 0.6, 0.5), 0.0))
    for a in range(-grid, grid):
        for b in range(-grid, grid):
            choose = rng.random()
            center = (a + 0.9 * rng.random(), 0.2, b + 0.9 * rng.random())
            if choose < 0.8:
                albedo = rng.random(3) * rng.random(3)
                m = s.lambertian(tuple(albedo))
            elif choose < 0.95:
                albedo = 0.5 + 0.5 * rng.random(3)
                m = s.metal(tuple(albedo), 0.5 * rng.random())
            else:
                m = s.dielectric(1.5)
            s.sphere(center, 0.2, m)
    s.camera = Camera(look_from=(13, 2, 3), look_at=(0, 0, 0), up=(0, 1, 0), vfov=20.0, aspect=16.0 / 9.0,
                      aperture=0.1, focus=10.0)
    if sky:
        s.set_background_sky()
    else:
        s.set_background_constant((0.70, 0.80, 1.00))
    return s


def spheres_params(**kw) -> RenderParams:
    p = dict(width=1280, height=720, spp=64, max_depth=50)
    p.update(kw)
    return RenderParams(**p)


def meshes(level=7, seed=DEFAULT_SEED, env_size=(2048, 1024), light=True) -> Scene:
    s = Scene(name="meshes")
    if light:
        # a hidden quad light above the instances, so the lambertian mixture PDF has a light to sample
        # (with an empty light list the reference's mixture PDF gives NaN / zero-direction bounces,
        # hittable_list.cuh:191-215, which would cut half the diffuse paths short)
        s.dir_light((0.0, 8.0, 1.0), (8.0, 0.0, 0.0), (0.0, 0.0, 4.0), (4.0, 4.0, 4.0), intensity=1.0, invisible=True)
    v, f = displaced_icosphere(level, 0.15, seed)
    mats = [s.metal((0.8, 0.85, 0.9), 0.05), s.dielectric(1.5), s.lambertian((0.7, 0.3, 0.2)),
            s.lambertian(s.image(procedural_image(512, 256, seed)))]
    xs = (-3.3, -1.1, 1.1, 3.3)
    uvs = sphere_uvs(v)
    for k, (x, m) in enumerate(zip(xs, mats)):
        # the fourth instance is image-textured through its per-vertex texture coordinates
        s.mesh((v + np.array([x, 1.0, 0.0])).astype(np.float32), f, m, uvs=uvs if k == 3 else None)
    ground = s.lambertian(s.checker_colors(10.0, (0.2, 0.3, 0.1), (0.9, 0.9, 0.9)))
    s.quad((-200.0, -0.15, -200.0), (400.0, 0.0, 0.0), (0.0, 0.0, 400.0), ground)
    s.camera = Camera(look_from=(0.0, 2.5, 9.0), look_at=(0.0, 0.9, 0.0), up=(0, 1, 0), vfov=35.0,
                      aspect=16.0 / 9.0, aperture=0.0, focus=9.0)
    s.set_background_env(sky_sun_envmap(*env_size))
    return s


def meshes_params(**kw) -> RenderParams:
    p = dict(width=1920, height=1080, spp=128, max_depth=16)
    p.update(kw)
    return RenderParams(**p)


def textured(seed=DEFAULT_SEED, floor_y=0.0) -> Scene:
    """Checker and image textures on spheres and quads, lit by a quad light and a sky.

    With the default floor_y = 0 the floor lies on a checker cell boundary (cells of 0.5 on every
    axis), so the floor's cell parity, floor(2 * hit_y), is decided by the sign of the hit point's
    rounding error - a rounding-level test of the texture path (bit-exact parity).  Convergence
    comparisons lift the floor off the boundary."""
    s = Scene(name="textured")
    s.dir_light((0.0, 8.0, 0.0), (4.0, 0.0, 0.0), (0.0, 0.0, 4.0), (6.0, 6.0, 6.0), intensity=1.0, invisible=True)
    img = s.image(procedural_image(64, 48, seed))
    chk = s.checker_colors(0.5, (0.2, 0.3, 0.1), (0.9, 0.9, 0.9))   # all_textures_spheres.scene scale style
    s.quad((-6.0, floor_y, -6.0), (12.0, 0.0, 0.0), (0.0, 0.0, 12.0), s.lambertian(chk))
    s.sphere((-1.6, 1.0, 0.0), 1.0, s.lambertian(img))
    s.sphere((1.6, 1.0, 0.0), 1.0, s.lambertian(s.checker_colors(0.3, (0.8, 0.1, 0.1), (0.9, 0.9, 0.2))))
    s.sphere((0.0, 0.6, 1.8), 0.6, s.metal((0.9, 0.9, 0.9), 0.2))
    s.quad((-3.0, 0.0, -3.0), (6.0, 0.0, 0.0), (0.0, 3.0, 0.0), s.lambertian(img))
    s.camera = Camera(look_from=(0.0, 3.0, 8.0), look_at=(0.0, 1.0, 0.0), up=(0, 1, 0), vfov=45.0, aspect=4.0 / 3.0,
                      aperture=0.0, focus=8.0)
    s.set_background_sky()
    return s


def icosphere_scene(level=3, seed=DEFAULT_SEED) -> Scene:
    s = Scene(name="icosphere")
    s.dir_light((0.0, 6.0, 0.0), (3.0, 0.0, 0.0), (0.0, 0.0, 3.0), (8.0, 8.0, 8.0), intensity=1.0, invisible=False)
    v, f = displaced_icosphere(level, 0.15, seed)
    mats = [s.lambertian((0.7, 0.3, 0.2)), s.metal((0.8, 0.8, 0.9), 0.1), s.dielectric(1.5)]
    for x, m in zip((-2.2, 0.0, 2.2), mats):
        s.mesh((v + np.array([x, 1.0, 0.0])).astype(np.float32), f, m)
    s.quad((-10.0, -0.2, -10.0), (20.0, 0.0, 0.0), (0.0, 0.0, 20.0), s.lambertian((0.5, 0.5, 0.5)))
    s.camera = Camera(look_from=(0.0, 2.5, 7.0), look_at=(0.0, 1.0, 0.0), up=(0, 1, 0), vfov=40.0, aspect=1.5,
                      aperture=0.05, focus=7.0)
    s.set_background_constant((0.3, 0.35, 0.45))
    return s


def uv_mesh_scene(seed=DEFAULT_SEED) -> Scene:
    """Image textures on triangle meshes through per-vertex texture coordinates: a displaced icosphere
    with an RGB8 image mapped by longitude/latitude, a second one whose coordinates wrap several times
    (values outside [0, 1) wrap as calculateTextureCoordinate does), and a metal mesh without texture
    coordinates beside them; a floor and a quad light."""
    s = Scene(name="uvmesh")
    s.dir_light((0.0, 6.0, 0.0), (3.0, 0.0, 0.0), (0.0, 0.0, 3.0), (8.0, 8.0, 8.0), intensity=1.0, invisible=True)
    v, f = displaced_icosphere(3, 0.15, seed)
    img = s.image(procedural_image(64, 48, seed))
    uvs = sphere_uvs(v)
    s.mesh((v + np.array([-2.2, 1.0, 0.0])).astype(np.float32), f, s.lambertian(img), uvs=uvs)
    s.mesh((v + np.array([0.0, 1.0, 0.0])).astype(np.float32), f, s.lambertian(img),
           uvs=(uvs * np.float32(3.0) - np.float32(1.25)).astype(np.float32))
    s.mesh((v + np.array([2.2, 1.0, 0.0])).astype(np.float32), f, s.metal((0.8, 0.8, 0.9), 0.1))
    s.quad((-10.0, -0.2, -10.0), (20.0, 0.0, 0.0), (0.0, 0.0, 20.0), s.lambertian((0.5, 0.5, 0.5)))
    s.camera = Camera(look_from=(0.0, 2.5, 7.0), look_at=(0.0, 1.0, 0.0), up=(0, 1, 0), vfov=40.0, aspect=1.5,
                      aperture=0.0, focus=7.0)
    s.set_background_constant((0.3, 0.35, 0.45))
    return s


def lights_scene(seed=DEFAULT_SEED) -> Scene:
    """Every light type: two omni lights (one hidden to primary rays), a directional quad light and a
    spot light cone, over lambertian, metal and dielectric spheres, a small displaced icosphere and a
    floor.  The light list is omni, omni, directional, spot, so light 0 (always the sampled one) is an
    omni light."""
    s = Scene(name="lights")
    s.omni_light((-2.5, 3.0, 1.0), 0.4, (6.0, 5.0, 4.0), intensity=1.5, invisible=True)
    s.omni_light((2.8, 2.2, -1.5), 0.3, (3.0, 4.0, 6.0), intensity=2.0, invisible=False)
    s.dir_light((0.0, 5.0, 0.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0), (4.0, 4.0, 4.0), intensity=1.0, invisible=True)
    s.spot_light((0.0, 3.5, 2.5), (0.0, -1.0, -0.6), 35.0, 4.0, (8.0, 8.0, 7.0), intensity=2.0, radius=0.25,
                 invisible=False)
    s.quad((-8.0, 0.0, -8.0), (16.0, 0.0, 0.0), (0.0, 0.0, 16.0), s.lambertian((0.6, 0.6, 0.6)))
    s.sphere((-1.5, 0.8, 0.0), 0.8, s.lambertian((0.8, 0.3, 0.2)))
    s.sphere((0.3, 0.6, 0.6), 0.6, s.metal((0.9, 0.9, 0.8), 0.15))
    s.sphere((1.6, 0.7, -0.4), 0.7, s.dielectric(1.5))
    v, f = displaced_icosphere(2, 0.1, seed)
    s.mesh((0.5 * v + np.array([0.0, 0.5, -2.0])).astype(np.float32), f, s.lambertian((0.2, 0.5, 0.8)))
    s.camera = Camera(look_from=(0.0, 2.2, 6.5), look_at=(0.0, 0.8, 0.0), up=(0, 1, 0), vfov=45.0, aspect=4.0 / 3.0,
                      aperture=0.0, focus=6.5)
    s.set_background_constant((0.02, 0.02, 0.03))
    return s


# -------------------------------------------------------------------------------------------------
# batched / served workload
# -------------------------------------------------------------------------------------------------
BATCH_RESOLUTIONS = [(256, 256), (512, 512), (768, 432), (1024, 1024)]
BATCH_SPP = [4, 16, 64]
_ICO_CACHE: dict = {}


def _mix_material(s: Scene, rng) -> int:
    """The ``spheres`` material mix: 80% lambertian (albedo U^3*U^3), 15% metal, 5% dielectric."""
    choose = rng.random()
    if choose < 0.8:
        return s.lambertian(tuple(rng.random(3) * rng.random(3)))
    if choose < 0.95:
        return s.metal(tuple(0.5 + 0.5 * rng.random(3)), 0.5 * rng.random())
    return s.dielectric(1.5)


def _cached_icosphere(level: int, seed: int):
    key = (level, seed)
    if key not in _ICO_CACHE:
        _ICO_CACHE[key] = displaced_icosphere(level, 0.15, seed)
    return _ICO_CACHE[key]


def batch_scene(k: int, seed=DEFAULT_SEED):
    """Scene `k` of the batched workload and its render parameters (see the module docstring)."""
    rng = np.random.default_rng([seed, k])
    target = math.exp(rng.uniform(math.log(1e3), math.log(5e5)))
    level, count = min(((lv, n) for lv in range(3, 8) for n in range(1, 5) if n * 20 * 4 ** lv <= 5e5),
                       key=lambda ln: abs(math.log(ln[1] * 20 * 4 ** ln[0] / target)))
    v, f = _cached_icosphere(level, seed)
    s = Scene(name=f"batch{k}")
    s.dir_light((0.0, 12.0, 0.0), (8.0, 0.0, 0.0), (0.0, 0.0, 8.0), (5.0, 5.0, 5.0), intensity=1.5, invisible=True)
    s.sphere((0.0, -1000.0, 0.0), 1000.0, s.lambertian((0.5, 0.5, 0.5)))
    for i in range(count):
        x = (i - (count - 1) / 2.0) * 2.4
        scale = 0.8 + 0.4 * rng.random()
        s.mesh((v * scale + np.array([x, scale * 1.15, 0.0])).astype(np.float32), f, _mix_material(s, rng))
    for _ in range(int(rng.integers(20, 121))):
        c = (rng.uniform(-7.0, 7.0), 0.2, rng.uniform(-7.0, 7.0))
        if abs(c[2]) < 1.6 and abs(c[0]) < 1.3 * count + 0.3:
            continue   # keep the instances' footprint clear
        s.sphere(c, 0.2, _mix_material(s, rng))
    w, h = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
    angle = rng.uniform(0.0, 2.0 * math.pi)
    dist = 10.0 + 2.0 * count
    s.camera = Camera(look_from=(dist * math.sin(angle), 3.0, dist * math.cos(angle)), look_at=(0.0, 1.0, 0.0),
                      up=(0, 1, 0), vfov=30.0, aspect=w / h, aperture=0.05, focus=dist)
    s.set_background_sky()
    params = RenderParams(width=w, height=h, spp=int(BATCH_SPP[int(rng.integers(len(BATCH_SPP)))]),
                          max_depth=int(rng.integers(8, 33)))
    return s, params


def batch_workload(n=64, seed=DEFAULT_SEED):
    """The batched workload: a list of (scene, params) for n scenes."""
    return [batch_scene(k, seed) for k in range(n)]


def orbit_camera(cam: Camera, angle: float, center=(0.0, 1.0, 0.0)) -> Camera:
    """`cam` rotated by `angle` radians about the vertical axis through `center` (served requests)."""
    f = np.asarray(cam.look_from, np.float64) - np.asarray(center, np.float64)
    ca, sa = math.cos(angle), math.sin(angle)
    r = np.array([ca * f[0] + sa * f[2], f[1], -sa * f[0] + ca * f[2]]) + np.asarray(center, np.float64)
    return Camera(look_from=tuple(r), look_at=tuple(center), up=cam.up, vfov=cam.vfov, aspect=cam.aspect,
                  aperture=cam.aperture, focus=cam.focus)


SCENES = {
    "cornell": (cornell, cornell_params),
    "spheres": (spheres, spheres_params),
    "meshes": (meshes, meshes_params),
    "textured": (textured, lambda **kw: RenderParams(**{**dict(width=160, height=120, spp=16, max_depth=10), **kw})),
    "icosphere": (icosphere_scene, lambda **kw: RenderParams(**{**dict(width=150, height=100, spp=16, max_depth=12), **kw})),
    "lights": (lights_scene, lambda **kw: RenderParams(**{**dict(width=120, height=90, spp=16, max_depth=10), **kw})),
    "uvmesh": (uv_mesh_scene, lambda **kw: RenderParams(**{**dict(width=120, height=80, spp=16, max_depth=10), **kw})),
    # boxes and transforms; "xforms" leaves out the multi-axis rotations the reference clips (see
    # transforms_scene), so the reference's own build renders it exactly
    "xforms": (lambda seed=DEFAULT_SEED: transforms_scene(seed, multi_axis=False), transforms_params),
    "xforms_multi": (transforms_scene, transforms_params),
}
