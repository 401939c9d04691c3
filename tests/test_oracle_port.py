"""Pins the oracle: the C restatement (oracle/rt_port.c) against the golden vectors produced by the
reference's own code (tests/golden/, made by tests/golden/make_golden.py from oracle/_ref/libref_cpu.so),
and the RNG known-answer tests (T0).  CPU only."""
import numpy as np
import pytest

from cortexraytracercuda_b200 import configs

import oracles
from golden.make_golden import GOLDEN_SCENES, golden_params, golden_rays

GOLD = oracles.ORACLE.parent / "tests" / "golden"


@pytest.fixture(scope="module")
def port():
    o = oracles.port()
    if o is None:
        import subprocess
        subprocess.run(["make", "-C", str(oracles.ORACLE), "port"], check=True, capture_output=True)
        o = oracles.port()
    assert o is not None
    return o


@pytest.fixture(scope="module")
def kat():
    return np.load(GOLD / "rng_kat.npz")


@pytest.fixture(scope="module")
def scenes():
    return np.load(GOLD / "scenes.npz")


def test_minstd_kat_python(kat):
    """thrust minstd_rand + uniform_real_distribution<float>: the Python restatement reproduces the
    reference's draws bit for bit."""
    for seed in (1984, 2580, 2580 + 65535):
        ref = kat[f"draws_{seed}"]
        assert np.array_equal(oracles.minstd_uniform(seed, 2000), ref[:2000])


def test_minstd_kat_port(port, kat):
    for seed in (1984, 2580, 2580 + 65535):
        assert np.array_equal(port.rng_draws(seed, 10000), kat[f"draws_{seed}"])


def test_uniform_reaches_one():
    """U = float(x-1) * 2^-31 rounds to exactly 1.0f for the largest states (thrust .inl:64-72)."""
    # x = m - 1 (the maximum state) is reached from seed s with 48271*s = m-1 (mod m): s = m - inv(48271)
    m = oracles.M31
    s = (m - pow(48271, -1, m)) % m
    assert oracles.minstd_uniform(s, 1)[0] == np.float32(1.0)


def test_get_int_is_min(kat):
    """get_int uses uniform_real_distribution<int>, whose integer division always yields `min`
    (gpu_randomizer.cuh:29-35)."""
    assert np.all(kat["get_int_2580_0_5"] == 0)


@pytest.mark.parametrize("which,name", [(0, "disk"), (1, "sphere"), (3, "light")])
def test_sampler_host_order(kat, which, name):
    """The g++ build evaluates multi-draw constructor/operator expressions right to left."""
    rep = oracles.sampler_reproduction(which, 2580, 500, 1)
    assert np.array_equal(rep, kat[f"sampler_{name}"])


def test_sphere_light_sampler_bitexact(port, kat):
    """omni_light::random (random_to_sphere with the reference's float M_PI) reproduced bit for bit."""
    assert np.array_equal(port.sphere_light_draws(2580, 500), kat["sampler_omni"])


def test_sampler_cosine_within_ulp(kat):
    rep = oracles.sampler_reproduction(2, 2580, 500, 1)
    ref = kat["sampler_cosine"]
    assert np.all(np.abs(rep - ref) <= np.spacing(np.abs(ref)) * 2)


@pytest.mark.parametrize("name", list(GOLDEN_SCENES))
def test_port_bitexact_vs_golden(port, scenes, name):
    mk, _ = configs.SCENES[name]
    p = golden_params(name)
    ps = port.scene(mk())
    pix = np.arange(p.width * p.height, dtype=np.int64)
    out, rays = ps.render_pixels(p, pix, threads=4, trig=0)
    ref = scenes[f"{name}_radiance"]
    st = oracles.parity_stats(out, ref)
    assert st["frac_exact"] == 1.0, st
    assert rays == int(scenes[f"{name}_rays"][0])


@pytest.mark.parametrize("name", list(GOLDEN_SCENES))
def test_port_hit_identity_vs_golden(port, scenes, name):
    mk, _ = configs.SCENES[name]
    ps = port.scene(mk())
    R = golden_rays(name)
    for depth, md in ((1, 1), (0, 8)):
        prim, t = ps.trace_closest(R, depth, md)
        ref = scenes[f"{name}_hit_{depth}_{md}_prim"]
        tref = scenes[f"{name}_hit_{depth}_{md}_t"]
        mism = prim != ref
        tie = mism & (t == tref)
        assert int((mism & ~tie).sum()) == 0
        same = prim == ref
        assert np.array_equal(t[same], tref[same])


def test_port_trig_mode_changes_only_last_bits(port):
    """trig=1 (double-rounded cos/sin) vs trig=0 (glibc): same image up to branch flips."""
    mk, _ = configs.SCENES["cornell"]
    p = golden_params("cornell")
    ps = port.scene(mk())
    pix = np.arange(p.width * p.height, dtype=np.int64)
    a, _ = ps.render_pixels(p, pix, threads=4, trig=0)
    b, _ = ps.render_pixels(p, pix, threads=4, trig=1)
    st = oracles.parity_stats(b, a)
    assert st["frac_ok"] >= 0.98 and st["mean_rel"] <= 0.02, st


@pytest.mark.parametrize("name,stride", [("cornell", 1), ("spheres", 29)])
def test_port_bitexact_vs_reference_full_size(port, name, stride):
    """The C restatement (glibc trig) against the reference's own g++ build at the measured frames' full
    sizes: the Cornell box at 256x256, 16 spp, depth 8 on every pixel, and the spheres frame at 1280x720,
    64 spp, depth 50 on every 29th pixel (a pixel's stream is its own, so a subsample is exact).  Every
    sampled pixel's FP32 sum is identical."""
    import os
    ref = oracles.ref_cpu()
    if ref is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    mk, mp = configs.SCENES[name]
    scene, p = mk(), mp()
    from cortexraytracercuda_b200.scene import DRAW_ORDER_HOST, MODE_COMPAT
    p.mode, p.draw_order = MODE_COMPAT, DRAW_ORDER_HOST
    pix = np.arange(0, p.width * p.height, stride, dtype=np.int64)
    threads = os.cpu_count() or 4
    ours, _ = port.scene(scene).render_pixels(p, pix, threads=threads, trig=0)
    theirs, _ = ref.scene(scene).render_pixels(p, pix, threads)
    st = oracles.parity_stats(ours, theirs)
    print(name, st)
    assert st["frac_exact"] == 1.0, st
