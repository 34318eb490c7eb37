"""The CPU reference of the albedo adjoint (oracle, double precision) against
central finite differences of the oracle's own renders: the derivative that
the GPU path-replay adjoint is checked against is itself checked here.

With Russian roulette off, a sample's radiance is a polynomial in a texel's
value (linear unless a path meets the texel twice), so the loss is a
low-order polynomial and a central difference with a large step is exact up
to its fourth-order term; a small step (1e-3) would be dominated by the FP32
rounding of the rendered image instead."""
import numpy as np

from mufflon_b200 import scenes

H_FD = 0.1


def _loss_and_render(oracle, tex, target, spp, seed=0):
    spec = scenes.cornell_box_textured(1, 24, 24, texture=tex)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=seed, max_path=5, nee_count=1, rr_start=5)
    for _ in range(spp):
        pt.iterate()
    img = pt.target("Radiance").astype(np.float64)
    return float(np.sum((img - target) ** 2)), img, pt


def test_oracle_adjoint_matches_finite_differences(oracle):
    rng = np.random.default_rng(3)
    tex = scenes.smooth_noise_texture(2, 8)
    target = rng.uniform(0.0, 0.5, (24, 24, 3))
    spp = 3
    loss, img, pt = _loss_and_render(oracle, tex, target, spp)
    grad = pt.albedo_gradient(0, spp, 2.0 * (img - target))
    assert np.abs(grad).max() > 0
    # the texels with the largest gradients, one channel each
    flat = np.argsort(-np.abs(grad).reshape(-1))[:6]
    for idx in flat:
        y, x, c = np.unravel_index(idx, grad.shape)
        tp, tm = tex.copy(), tex.copy()
        tp[y, x, c] += H_FD
        tm[y, x, c] -= H_FD
        lp, _, _ = _loss_and_render(oracle, tp, target, spp)
        lm, _, _ = _loss_and_render(oracle, tm, target, spp)
        fd = (lp - lm) / (2 * H_FD)
        assert abs(fd - grad[y, x, c]) <= 1e-3 * abs(grad[y, x, c]) + 1e-6, (y, x, c, fd, grad[y, x, c])


def test_oracle_adjoint_rejects_russian_roulette(oracle):
    spec = scenes.cornell_box_textured(1, 8, 8, texture_size=4)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), max_path=5, rr_start=0)
    try:
        pt.albedo_gradient(0, 1, np.zeros((8, 8, 3), np.float32))
    except ValueError:
        return
    raise AssertionError("expected a rejection")


def _emission_loss(oracle, radiance, target, spp, rr_start):
    spec = scenes.cornell_box(1, 24, 24)
    mats = list(spec.materials)
    li = [i for i, m in enumerate(mats) if m.type == scenes.MAT_EMISSIVE][0]
    mats[li] = scenes.MaterialSpec(scenes.MAT_EMISSIVE, radiance=tuple(radiance), name="light")
    import dataclasses
    spec = dataclasses.replace(spec, materials=mats)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), seed=0, max_path=6, nee_count=1, rr_start=rr_start)
    for _ in range(spp):
        pt.iterate()
    img = pt.target("Radiance").astype(np.float64)
    return float(np.sum((img - target) ** 2)), img, pt, li


def test_oracle_emission_adjoint_matches_finite_differences(oracle):
    """The Cornell box has one area light, so its selection probability does not depend on its
    radiance and the image is linear in it (Russian roulette on or off): the loss is quadratic and
    a central difference with a large step is exact up to FP32 rounding of the render."""
    rng = np.random.default_rng(5)
    target = rng.uniform(0.0, 0.5, (24, 24, 3))
    L = np.array([15.0, 12.0, 9.0])
    for rr_start in (0, 6):
        loss, img, pt, li = _emission_loss(oracle, L, target, 3, rr_start)
        grad = pt.emission_gradient(li, 3, 2.0 * (img - target))
        assert np.all(np.abs(grad) > 0)
        for c in range(3):
            lp = L.copy(); lp[c] += 1.0
            lm = L.copy(); lm[c] -= 1.0
            fd = (_emission_loss(oracle, lp, target, 3, rr_start)[0] - _emission_loss(oracle, lm, target, 3, rr_start)[0]) / 2.0
            assert abs(fd - grad[c]) <= 1e-4 * abs(grad[c]), (rr_start, c, fd, grad[c])


def test_oracle_emission_adjoint_rejects_non_emitters(oracle):
    spec = scenes.cornell_box(1, 8, 8)
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec), max_path=4)
    try:
        pt.emission_gradient(0, 1, np.zeros((8, 8, 3), np.float32))  # a Lambert material
    except ValueError:
        return
    raise AssertionError("expected a rejection")
