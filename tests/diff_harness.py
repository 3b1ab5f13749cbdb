"""Test-harness wrapper of the renderer's differentiable pair
(render_batch with path records, render_backward) as a torch.autograd.Function.

Only the tests use it: the library's boundary is the C ABI."""
import numpy as np
import torch

import ymrt_b200 as Y


class MultiViewRenderer:
    """Several views (scenes that share one material table), rendered together."""

    def __init__(self, ctx, scenes, setting, frame_index=1):
        self.ctx, self.scenes, self.setting, self.frame = ctx, scenes, setting, frame_index
        self.images = [torch.zeros((s.height, s.width, 4), dtype=torch.float32, device="cuda") for s in scenes]
        self.renders = [[s, setting, frame_index, img] for s, img in zip(scenes, self.images)]
        self.records = [torch.zeros((Y.path_count(r), 4), dtype=torch.float32, device="cuda") for r in self.renders]
        self.n_materials = scenes[0].material_params().shape[0]

    def set_params(self, params: np.ndarray):
        for s in self.scenes:
            s.set_material_params(params)

    def forward(self):
        st = Y.render_batch(self.ctx, self.renders, self.records)
        assert st.device_errors == 0
        return [img.clone() for img in self.images]

    def backward(self, dlosses):
        grads = torch.zeros((self.n_materials, 4), dtype=torch.float32, device="cuda")
        dl = [d.contiguous() for d in dlosses]
        st = Y.render_backward(self.ctx, self.renders, self.records, dl, grads)
        assert st.device_errors == 0
        return grads


class RenderFunction(torch.autograd.Function):
    """images = render(params); params: (materials, 4) albedo rgb + roughness."""

    @staticmethod
    def forward(fctx, params, renderer):
        renderer.set_params(params.detach().cpu().numpy())
        fctx.renderer = renderer
        fctx.param_device, fctx.param_dtype = params.device, params.dtype
        return torch.stack(renderer.forward())

    @staticmethod
    def backward(fctx, grad_images):
        grads = fctx.renderer.backward([g for g in grad_images])
        return grads.to(device=fctx.param_device, dtype=fctx.param_dtype), None
