"""Differentiable rendering of an albedo texture and of emitted radiance
through torch.autograd.

The forward pass renders the loaded scenario (spp iterations after a reset)
with the texture's texels replaced by the input tensor; the backward pass
computes dLoss/dTexel from dLoss/dImage with the library's path-replay adjoint
(mufflon_albedo_gradient), which replays the same samples from the same seed.
Russian roulette is switched off (RR start depth = max path length), which
makes the rendered image a smooth (polynomial) function of the texels.

    r = AlbedoRenderer(dll, dll.textures[0], (512, 512), spp=16, max_path=6)
    tex = torch.full((512, 512, 3), 0.5, requires_grad=True)
    loss = ((render_albedo(tex, r) - target) ** 2).sum()
    loss.backward()            # tex.grad = dLoss/dTexel

The emitted radiance L (radiance x scale, RGB) of an emissive material works
the same way (mufflon_emission_gradient); the image is linear in L, and
Russian roulette may stay on:

    e = EmissionRenderer(dll, dll.materials[5], spp=16, max_path=6)
    L = torch.tensor([15.0, 15.0, 15.0], requires_grad=True)
    loss = ((render_emission(L, e) - target) ** 2).sum()
    loss.backward()            # L.grad = dLoss/dL
"""
from __future__ import annotations

import numpy as np


class AlbedoRenderer:
    """Renders `dll`'s loaded scenario as a function of albedo texture `texture`."""

    def __init__(self, dll, texture, tex_shape, spp: int, seed: int = 0, max_path: int = 6, nee: int = 1):
        self.dll, self.texture, self.tex_shape = dll, texture, tuple(tex_shape[:2])
        self.spp = int(spp)
        for name, v in {"Seed": seed, "Max. path length": max_path, "Min. path length": 0, "NEE count": nee,
                        "RR start depth": max_path}.items():
            if not dll.renderer_set_parameter_int(name, v):
                raise ValueError(f"cannot set {name}")
        dll.render_enable_render_target("Radiance", False)
        self.last_forward_ms = 0.0
        self.last_adjoint_ms = 0.0

    def render(self, texels: np.ndarray) -> np.ndarray:
        t = np.asarray(texels, np.float32)
        if t.shape[:2] != self.tex_shape:
            raise ValueError(f"texture shape {t.shape} != {self.tex_shape}")
        self.dll.texture_update(self.texture, t)
        self.dll.render_reset()
        ms = 0.0
        for _ in range(self.spp):
            self.dll.render_iterate()
            ms += self.dll.render_stats()["kernelMs"]
        self.last_forward_ms = ms
        return self.dll.get_target_image("Radiance").copy()

    def gradient(self, image_grad: np.ndarray) -> np.ndarray:
        g, ms = self.dll.albedo_gradient(self.texture, self.spp, image_grad, self.tex_shape)
        self.last_adjoint_ms = ms
        return g


class EmissionRenderer:
    """Renders `dll`'s loaded scenario as a function of the emitted radiance of emissive `material`."""

    def __init__(self, dll, material, spp: int, seed: int = 0, max_path: int = 6, nee: int = 1, rr_start: int = 0):
        self.dll, self.material, self.spp = dll, material, int(spp)
        for name, v in {"Seed": seed, "Max. path length": max_path, "Min. path length": 0, "NEE count": nee,
                        "RR start depth": rr_start}.items():
            if not dll.renderer_set_parameter_int(name, v):
                raise ValueError(f"cannot set {name}")
        dll.render_enable_render_target("Radiance", False)
        self.last_forward_ms = 0.0
        self.last_adjoint_ms = 0.0

    def render(self, radiance: np.ndarray) -> np.ndarray:
        self.dll.set_emitted_radiance(self.material, np.asarray(radiance, np.float32))
        self.dll.render_reset()
        ms = 0.0
        for _ in range(self.spp):
            self.dll.render_iterate()
            ms += self.dll.render_stats()["kernelMs"]
        self.last_forward_ms = ms
        return self.dll.get_target_image("Radiance").copy()

    def gradient(self, image_grad: np.ndarray) -> np.ndarray:
        g, ms = self.dll.emission_gradient(self.material, self.spp, image_grad)
        self.last_adjoint_ms = ms
        return g


try:
    import torch

    class RenderAlbedo(torch.autograd.Function):
        @staticmethod
        def forward(ctx, texels, renderer):
            img = renderer.render(texels.detach().to("cpu", torch.float32).numpy())
            ctx.renderer = renderer
            return torch.from_numpy(img).to(texels.device)

        @staticmethod
        def backward(ctx, grad_image):
            g = ctx.renderer.gradient(grad_image.detach().to("cpu", torch.float32).contiguous().numpy())
            return torch.from_numpy(g).to(grad_image.device), None

    def render_albedo(texels, renderer):
        """Image (H, W, 3) rendered with albedo texels (H_t, W_t, 3), differentiable in the texels."""
        return RenderAlbedo.apply(texels, renderer)

    class RenderEmission(torch.autograd.Function):
        @staticmethod
        def forward(ctx, radiance, renderer):
            img = renderer.render(radiance.detach().to("cpu", torch.float32).numpy())
            ctx.renderer = renderer
            return torch.from_numpy(img).to(radiance.device)

        @staticmethod
        def backward(ctx, grad_image):
            g = ctx.renderer.gradient(grad_image.detach().to("cpu", torch.float32).contiguous().numpy())
            return torch.from_numpy(g).to(grad_image.device), None

    def render_emission(radiance, renderer):
        """Image (H, W, 3) rendered with emitted radiance (3,) of the renderer's material, differentiable in it."""
        return RenderEmission.apply(radiance, renderer)
except ImportError:  # torch is optional for the C-level API
    pass
