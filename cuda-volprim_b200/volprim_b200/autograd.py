"""torch.autograd.Function over the hand-written adjoint (vp_render_emission_backward).

    images = render_emission_images(mean, log_scale, quat_wxyz, density, emission,
                                    cameras, config, env, sigma_multiplier=1.0)

returns (n_cameras, H, W, 3) absorption-plus-emission images (the model of
include/volprim_b200.h) that are differentiable with respect to the five parameter tensors.  The
forward pass builds the scene (LBVH + BVH32 from the current parameters) on the device and
renders each camera; the backward pass traverses every ray again and adds the per-Gaussian
gradients of all cameras.  PyTorch is only the plumbing here: both passes are the library's
CUDA kernels.
"""
from __future__ import annotations

from typing import Sequence

import torch

from .api import Camera, Config, Context, Environment, Gaussians, Scene
from .emission import render_emission, render_emission_backward


class EmissionRender(torch.autograd.Function):
    # Device times of the most recent forward (scene build, forward kernels) and backward (adjoint
    # kernels) in milliseconds, from the library's CUDA events.
    last_ms = {"scene_build": 0.0, "forward_kernels": 0.0, "backward_kernels": 0.0}

    @staticmethod
    def forward(ctx, mean, log_scale, quat_wxyz, density, emission, cameras, config, env, sigma_multiplier, vp_ctx):
        dev = mean.device
        scene = Scene(vp_ctx, Gaussians(mean.detach(), log_scale.detach(), quat_wxyz.detach(), density.detach(),
                                        scale_is_log=True), sigma_multiplier)
        scene.set_emission(emission.detach())
        H, W = config.image_height, config.image_width
        imgs = torch.empty((len(cameras), H, W, 4), dtype=torch.float32, device=dev)
        fwd_ms = 0.0
        for k, cam in enumerate(cameras):
            st = {}
            render_emission(scene, env, cam, config, out=imgs[k], stats=st)
            fwd_ms += st.get("ms_kernels", 0.0)
        EmissionRender.last_ms = {"scene_build": scene.info()["build_ms"], "forward_kernels": fwd_ms,
                                  "backward_kernels": 0.0}
        ctx.scene, ctx.cameras, ctx.config, ctx.env = scene, list(cameras), config, env
        ctx.shapes = (mean.shape, log_scale.shape, quat_wxyz.shape, density.shape, emission.shape)
        return imgs[..., :3].clone()

    @staticmethod
    def backward(ctx, grad_images):
        dev = grad_images.device
        n = ctx.shapes[3][0]
        grads = {"mean": torch.zeros(3 * n, dtype=torch.float32, device=dev),
                 "scale": torch.zeros(3 * n, dtype=torch.float32, device=dev),
                 "quat_wxyz": torch.zeros(4 * n, dtype=torch.float32, device=dev),
                 "density": torch.zeros(n, dtype=torch.float32, device=dev),
                 "emission": torch.zeros(3 * n, dtype=torch.float32, device=dev)}
        H, W = ctx.config.image_height, ctx.config.image_width
        dl = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
        bwd_ms = 0.0
        for k, cam in enumerate(ctx.cameras):
            dl[..., :3] = grad_images[k]
            bwd_ms += render_emission_backward(ctx.scene, ctx.env, cam, ctx.config, dl, grads).get("ms_kernels", 0.0)
        EmissionRender.last_ms["backward_kernels"] = bwd_ms
        ctx.scene.close()
        out = [grads["mean"].view(ctx.shapes[0]), grads["scale"].view(ctx.shapes[1]),
               grads["quat_wxyz"].view(ctx.shapes[2]), grads["density"].view(ctx.shapes[3]),
               grads["emission"].view(ctx.shapes[4])]
        return (*out, None, None, None, None, None)


def render_emission_images(mean, log_scale, quat_wxyz, density, emission, cameras: Sequence[Camera],
                           config: Config, env: Environment, sigma_multiplier: float = 1.0,
                           vp_ctx: Context | None = None):
    if vp_ctx is None:
        vp_ctx = env.ctx
    return EmissionRender.apply(mean, log_scale, quat_wxyz, density, emission, tuple(cameras), config, env,
                                float(sigma_multiplier), vp_ctx)
