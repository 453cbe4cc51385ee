"""Differentiable rendering harness: xyzgpu_render / xyzgpu_adjoint behind a
torch.autograd.Function.

The parameters are the materials' 3-channel albedo (n_materials, 3) and
emission scale (n_materials,); the output is the image (H, W, 3), the film's
mean over samples.  The backward pass is the library's path-replay adjoint
(xyzgpu_adjoint): it replays `adjoint_spp` sample paths starting at sample
`adjoint_offset` (0 = the primal's own samples, so the gradient is the exact
derivative of the rendered image; spp = the primal's next samples, so the
gradient is an independent unbiased estimate).  Russian roulette is off by
default (rr_threshold 0), which makes the rendered image a polynomial in the
parameters with no discontinuities: central finite differences of the same
render converge to the adjoint's gradient.

This is the thin harness around the C ABI; the kernels, the path replay and the
gradient accumulation are all in libxyzgpu.so.
"""

from __future__ import annotations

import torch

from . import api


class Renderer:
    """A scene, camera and sample budget; calling it renders an image that
    autograd can differentiate with respect to (albedo, emission)."""

    def __init__(self, scene: api.Scene, camera, width: int, height: int, spp: int, *,
                 adjoint_spp: int | None = None, adjoint_offset: int | None = None, seed: int = 0,
                 max_depth: int = 6, rr_threshold: float = 0.0):
        self.scene = scene
        self.camera = camera
        self.width, self.height = width, height
        self.spp = spp
        self.adjoint_spp = spp if adjoint_spp is None else adjoint_spp
        self.adjoint_offset = spp if adjoint_offset is None else adjoint_offset
        self.seed = seed
        self.max_depth = max_depth
        self.rr_threshold = rr_threshold

    def render(self, spp: int | None = None, spp_offset: int = 0) -> torch.Tensor:
        """Image (H, W, 3) of the current materials: film / spp."""
        spp = self.spp if spp is None else spp
        film = self.scene.render(self.camera, self.width, self.height, spp, seed=self.seed,
                                 spp_offset=spp_offset, max_depth=self.max_depth,
                                 rr_threshold=self.rr_threshold)
        return film / float(spp)

    def gradient(self, d_image: torch.Tensor):
        """(d_albedo, d_emission) of sum(d_image * image) for the current
        materials, by the adjoint over the replay samples."""
        d_film = (d_image / float(self.adjoint_spp)).contiguous()
        return self.scene.adjoint(self.camera, self.width, self.height, self.adjoint_spp, d_film,
                                  seed=self.seed, spp_offset=self.adjoint_offset,
                                  max_depth=self.max_depth, rr_threshold=self.rr_threshold)

    def __call__(self, albedo: torch.Tensor, emission: torch.Tensor) -> torch.Tensor:
        return RenderFunction.apply(albedo, emission, self)


class RenderFunction(torch.autograd.Function):
    """image = render(albedo, emission); backward = path-replay adjoint."""

    @staticmethod
    def forward(ctx, albedo, emission, renderer: Renderer):
        a = albedo.detach().to(torch.float32).contiguous()
        e = emission.detach().to(torch.float32).contiguous()
        renderer.scene.set_materials(a, e)
        ctx.renderer = renderer
        ctx.save_for_backward(a, e)
        return renderer.render()

    @staticmethod
    def backward(ctx, grad_image):
        r = ctx.renderer
        a, e = ctx.saved_tensors
        r.scene.set_materials(a, e)
        d_albedo, d_emission = r.gradient(grad_image.to(torch.float32))
        return d_albedo, d_emission, None
