"""Test-only PyTorch binding of the differentiable SBS render (over the C-ABI
lrt_sbs_update_values / lrt_render_lambert / lrt_adjoint_lambert_sbs, or
their image-order forms when image_size = (width, height) is given).

    img = SbsLambertRender.apply(values_f, scene, rays, light[, image_size])
    loss = ((img - target) ** 2).mean()
    loss.backward()            # values_f.grad from the adjoint sphere tracer

values_f is the scene's whole SBS float array (torch CUDA tensor); forward
uploads it, renders the Lambert image of `rays` (CUDA float32, n x 8) and
backward runs the adjoint kernel with the incoming image gradient.  The scene
must not be changed between forward and backward.
"""
import torch


class SbsLambertRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values_f, scene, rays, light, image_size=None):
        values_f = values_f.detach().contiguous()
        n = rays.numel() // 8
        scene.update_sbs_values(values_f.data_ptr(), values_f.numel(), device=True)
        img = torch.empty(n, dtype=torch.float32, device=rays.device)
        scene.render_lambert(rays.data_ptr(), n, light, img.data_ptr(), image_size=image_size)
        scene.sync()
        ctx.scene, ctx.light, ctx.n, ctx.image_size = scene, light, n, image_size
        ctx.save_for_backward(rays, values_f)
        return img

    @staticmethod
    def backward(ctx, grad_img):
        rays, values_f = ctx.saved_tensors
        grad = torch.zeros_like(values_f)
        g = grad_img.detach().contiguous().to(torch.float32)
        ctx.scene.adjoint_lambert(rays.data_ptr(), ctx.n, ctx.light, g.data_ptr(), grad.data_ptr(),
                                  image_size=ctx.image_size)
        ctx.scene.sync()
        return grad, None, None, None, None
