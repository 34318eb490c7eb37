"""Path-replay adjoint of the albedo texture on the GPU: against the oracle's
double-precision gradient, against central differences of GPU renders, and
through torch.autograd."""
import numpy as np
import pytest

from mufflon_b200 import bindings, scenes

pytestmark = pytest.mark.gpu

W = 32
TEX = 16
SPP = 4
DEPTH = 5
H_FD = 0.1  # central difference of a low-order polynomial (see tests/test_oracle_adjoint.py)


@pytest.fixture(scope="module")
def world():
    tex = scenes.smooth_noise_texture(5, TEX)
    spec = scenes.cornell_box_textured(2, W, W, texture=tex)
    d = bindings.DllInterface()
    bindings.load_scene_spec(d, spec)
    assert d.render_enable_renderer(0, 0)
    yield d, spec, tex
    d.close()


def _renderer(d):
    from mufflon_b200.adjoint import AlbedoRenderer
    return AlbedoRenderer(d, d.textures[0], (TEX, TEX), spp=SPP, seed=1, max_path=DEPTH)


def _target():
    return np.random.default_rng(11).uniform(0.0, 0.4, (W, W, 3)).astype(np.float32)


def test_forward_matches_oracle(world, oracle):
    d, spec, tex = world
    r = _renderer(d)
    img = r.render(tex[..., :3])
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=1, max_path=DEPTH, rr_start=DEPTH)
    for _ in range(SPP):
        pt.iterate()
    ref = pt.target("Radiance")
    assert np.sqrt(np.mean((img - ref) ** 2)) <= 1e-4 * np.sqrt(np.mean(ref ** 2))


@pytest.mark.parametrize("megakernel", [0, 1])
def test_gradient_matches_fp64_oracle(world, oracle, megakernel):
    """Both adjoint schedules: through the wavefront kernels (default) and one thread per path."""
    d, spec, tex = world
    assert d.renderer_set_parameter_int("Megakernel", megakernel)
    r = _renderer(d)
    target = _target()
    img = r.render(tex[..., :3])
    dldi = 2.0 * (img - target)
    g = r.gradient(dldi)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=1, max_path=DEPTH, rr_start=DEPTH)
    ref = pt.albedo_gradient(0, SPP, dldi)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(g - ref).max() <= 1e-4 * scale
    big = np.abs(ref) > 1e-2 * scale
    assert np.all(np.abs(g[big] - ref[big]) <= 1e-3 * np.abs(ref[big]))
    assert d.renderer_set_parameter_int("Megakernel", 0)


def test_gradient_matches_central_differences(world):
    d, spec, tex = world
    r = _renderer(d)
    target = _target()
    t0 = tex[..., :3].copy()
    g = r.gradient(2.0 * (r.render(t0) - target))
    loss = lambda t: float(np.sum((r.render(t).astype(np.float64) - target) ** 2))
    idx = np.argsort(-np.abs(g).reshape(-1))[:64]  # 64 texel channels with the largest gradients
    for k in idx:
        y, x, c = np.unravel_index(k, g.shape)
        tp, tm = t0.copy(), t0.copy()
        tp[y, x, c] += H_FD
        tm[y, x, c] -= H_FD
        fd = (loss(tp) - loss(tm)) / (2 * H_FD)
        assert abs(fd - g[y, x, c]) <= 1e-3 * abs(g[y, x, c]) + 1e-5, (y, x, c, fd, g[y, x, c])


def test_torch_autograd(world):
    import torch
    from mufflon_b200.adjoint import render_albedo
    d, spec, tex = world
    r = _renderer(d)
    target = torch.from_numpy(_target())
    t = torch.tensor(tex[..., :3], requires_grad=True)
    loss = ((render_albedo(t, r) - target) ** 2).sum()
    loss.backward()
    img = r.render(tex[..., :3])
    direct = r.gradient(2.0 * (img - target.numpy()))
    assert np.allclose(t.grad.numpy(), direct, rtol=1e-5, atol=1e-7)
    assert r.last_adjoint_ms > 0


def test_gradient_requires_roulette_off(world):
    d, spec, tex = world
    assert d.renderer_set_parameter_int("RR start depth", 0)
    with pytest.raises(bindings.MufflonError):
        d.albedo_gradient(d.textures[0], 1, np.zeros((W, W, 3), np.float32), (TEX, TEX))


# ---------------------------------------------------------------- emission
# The gradient with respect to the emitted radiance L (radiance x scale) of
# the Cornell box's ceiling light. The scene has one area light, so its
# selection probability does not depend on L and the image is linear in L,
# with Russian roulette on or off: a central difference is exact for any
# step up to the FP32 rounding of the rendered image.
L0 = np.array([15.0, 12.0, 9.0], np.float32)


@pytest.fixture(scope="module")
def emitter_world():
    spec = scenes.cornell_box(4, W, W)
    li = [i for i, m in enumerate(spec.materials) if m.type == scenes.MAT_EMISSIVE][0]
    d = bindings.DllInterface()
    bindings.load_scene_spec(d, spec)
    assert d.render_enable_renderer(0, 0)
    yield d, spec, li
    d.close()


def _emission_renderer(d, li, rr_start):
    from mufflon_b200.adjoint import EmissionRenderer
    return EmissionRenderer(d, d.materials[li], spp=SPP, seed=2, max_path=DEPTH + 1, rr_start=rr_start)


def _oracle_with_emission(oracle, spec, li, L, rr_start):
    import dataclasses
    mats = list(spec.materials)
    mats[li] = scenes.MaterialSpec(scenes.MAT_EMISSIVE, radiance=tuple(float(x) for x in L), name="light")
    spec = dataclasses.replace(spec, materials=mats)
    return oracle.OraclePathTracer(oracle.OracleScene(spec), seed=2, max_path=DEPTH + 1, rr_start=rr_start)


@pytest.mark.parametrize("rr_start", [0, DEPTH + 1], ids=["roulette", "no_roulette"])
@pytest.mark.parametrize("megakernel", [0, 1], ids=["wavefront", "megakernel"])
def test_emission_gradient_matches_fp64_oracle(emitter_world, oracle, megakernel, rr_start):
    d, spec, li = emitter_world
    assert d.renderer_set_parameter_int("Megakernel", megakernel)
    e = _emission_renderer(d, li, rr_start)
    img = e.render(L0)
    pt = _oracle_with_emission(oracle, spec, li, L0, rr_start)
    for _ in range(SPP):
        pt.iterate()
    ref_img = pt.target("Radiance")
    assert np.sqrt(np.mean((img - ref_img) ** 2)) <= 1e-4 * np.sqrt(np.mean(ref_img ** 2))
    dldi = 2.0 * (img - _target())
    g = e.gradient(dldi)
    ref = pt.emission_gradient(li, SPP, dldi)
    assert np.all(np.abs(ref) > 0)
    assert np.all(np.abs(g - ref) <= 1e-4 * np.abs(ref)), (g, ref)
    assert d.renderer_set_parameter_int("Megakernel", 0)


@pytest.mark.parametrize("h", [1e-3, 1.0])
def test_emission_gradient_matches_central_differences(emitter_world, h):
    d, spec, li = emitter_world
    e = _emission_renderer(d, li, 0)
    target = _target()
    g = e.gradient(2.0 * (e.render(L0) - target))
    loss = lambda L: float(np.sum((e.render(L).astype(np.float64) - target) ** 2))
    for c in range(3):
        lp, lm = L0.copy(), L0.copy()
        lp[c] += h
        lm[c] -= h
        fd = (loss(lp) - loss(lm)) / (2 * h)
        # h = 1e-3 changes the image by ~1e-4 of itself, so its FP32 rounding (~1e-7) bounds the
        # quotient's accuracy near 1e-3; with h = 1 the quotient is exact to ~1e-6
        tol = 2e-3 if h < 0.01 else 1e-4
        assert abs(fd - g[c]) <= tol * abs(g[c]), (c, h, fd, g[c])


def test_emission_torch_autograd(emitter_world):
    import torch
    from mufflon_b200.adjoint import render_emission
    d, spec, li = emitter_world
    e = _emission_renderer(d, li, 0)
    target = torch.from_numpy(_target())
    L = torch.tensor(L0, requires_grad=True)
    loss = ((render_emission(L, e) - target) ** 2).sum()
    loss.backward()
    direct = e.gradient(2.0 * (e.render(L0) - target.numpy()))
    assert np.allclose(L.grad.numpy(), direct, rtol=1e-5)
    assert e.last_adjoint_ms > 0


def test_emission_gradient_rejects_non_emitters(emitter_world):
    d, spec, li = emitter_world
    with pytest.raises(bindings.MufflonError, match="not emissive"):
        d.emission_gradient(d.materials[0], 1, np.zeros((W, W, 3), np.float32))
