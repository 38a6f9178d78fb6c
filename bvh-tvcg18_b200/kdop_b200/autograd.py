"""torch.autograd wrapper of contact generation and its hand-written adjoint.

ContactGeometry.apply(xyz, scene, pairs) runs refit + tandem traversal +
MOST_OPPOSING contact generation on the world vertex positions `xyz` (a CUDA
float32 tensor, all meshes of the scene concatenated) and returns per-contact
depth (n,) and normal (n, 3) tensors plus the contact rows.  Its backward
calls the adjoint kernel (kdop_contacts_adjoint), which carries dL/d(depth)
and dL/d(normal) back to the vertex positions with the candidate pair set and
every discrete choice of the forward pass (contact face, extreme candidates)
held fixed.
"""
from __future__ import annotations

import numpy as np
import torch

from . import lib as kd


class ContactGeometry(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz: torch.Tensor, scene: "kd.DeviceScene", pairs, opts=None):
        if not xyz.is_cuda or xyz.dtype != torch.float32:
            raise TypeError("xyz must be a float32 CUDA tensor")
        torch.cuda.current_stream().synchronize()
        scene.set_vertices(xyz.detach().contiguous())
        scene.refit(kd.REFIT_VERTICES)
        scene.traverse_sync(pairs, opts, contacts=True)
        rows = scene.read_contacts()
        depth = torch.from_numpy(np.ascontiguousarray(rows["depth"])).to(xyz.device)
        normal = torch.from_numpy(np.ascontiguousarray(rows["n"])).to(xyz.device)
        ctx.scene = scene
        ctx.n_verts = xyz.shape[0]
        return depth, normal

    @staticmethod
    def backward(ctx, g_depth, g_normal):
        scene = ctx.scene
        dev = g_depth.device if g_depth is not None else g_normal.device
        n = scene.stats(check=False).n_contacts
        gd = (g_depth if g_depth is not None else torch.zeros(n, device=dev)).float().contiguous()
        gn = (g_normal if g_normal is not None else torch.zeros((n, 3), device=dev)).float().contiguous()
        grad = torch.zeros((ctx.n_verts, 3), dtype=torch.float32, device=dev)
        torch.cuda.current_stream().synchronize()
        scene.adjoint(gd, gn, grad)
        scene.ctx.synchronize()
        return grad, None, None, None


def contact_geometry(xyz: torch.Tensor, scene: "kd.DeviceScene", pairs, opts=None):
    """(depth, normal) of every contact, differentiable in xyz."""
    return ContactGeometry.apply(xyz, scene, pairs, opts)
