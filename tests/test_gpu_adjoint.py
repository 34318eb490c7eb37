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
