"""torch.autograd binding of the docking energy at fixed poses.

`docking_energy(batch, pose_ligand, poses, weights)` returns the energy of each
pose (model::eval_deriv's inter + intra energy, unidock/src/lib/model.cpp:935-962,
with curl caps v_intra / v_inter) as a differentiable function of

  * the pose DOFs [x y z qw qx qy qz t0 .. t(T-1)] (the orientation enters as
    q / |q|, so any non-zero quaternion is accepted), and
  * the scoring-term weights (reference order, e.g. Vina gauss1, gauss2,
    repulsion, hydrophobic, hbond, glue).

The forward pass runs the adjoint kernel for energies only; the backward pass
runs it again, recomputing the conformer from the pose, for the pose-layout
gradient and the term-weight gradient (ud_score_adjoint_device).  Weights
that differ from the maps' current ones are applied with ud_maps_set_weights,
which rebuilds the maps and tables on the GPU as weight-sums of per-term data.
There is no CPU path: without the CUDA library this raises.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _apply_weights(batch, w):
    if w is None:
        return
    cur = batch.maps.weights()
    if not np.array_equal(cur, w):
        batch.maps.set_weights(w, stream=_stream())


class DockingEnergy(torch.autograd.Function):
    """Energy per pose; gradients for `poses` and `weights` (see module doc)."""

    @staticmethod
    def forward(ctx, poses, weights, batch, pose_ligand, v_intra, v_inter, exact):
        if not poses.is_cuda or poses.dtype != torch.float32:
            raise TypeError("poses must be a float32 CUDA tensor")
        poses = poses.contiguous()
        pose_ligand = pose_ligand.to(device=poses.device, dtype=torch.int32).contiguous()
        n, stride = poses.shape
        w = None if weights is None else weights.detach().to("cpu", torch.float32).numpy().copy()
        _apply_weights(batch, w)
        e = torch.empty(n, dtype=torch.float32, device=poses.device)
        if n:
            batch.score_adjoint_device(pose_ligand.data_ptr(), poses.data_ptr(), n, stride, e.data_ptr(),
                                       v_intra=v_intra, v_inter=v_inter, exact=exact, stream=_stream())
        ctx.save_for_backward(poses, pose_ligand)
        ctx.batch, ctx.w, ctx.v = batch, w, (v_intra, v_inter, exact)
        ctx.want_w = weights is not None
        ctx.w_like = (weights.device, weights.dtype) if weights is not None else None
        return e

    @staticmethod
    def backward(ctx, grad_e):
        poses, pose_ligand = ctx.saved_tensors
        batch = ctx.batch
        v_intra, v_inter, exact = ctx.v
        n, stride = poses.shape
        _apply_weights(batch, ctx.w)  # another forward may have changed them since
        gs = 7 + batch.max_torsions
        nt = batch.maps.n_terms
        need_w = ctx.want_w and ctx.needs_input_grad[1]
        e = torch.empty(n, dtype=torch.float32, device=poses.device)
        g = torch.zeros((n, gs), dtype=torch.float32, device=poses.device)
        dw = torch.zeros((n, nt), dtype=torch.float32, device=poses.device) if need_w else None
        if n:
            batch.score_adjoint_device(pose_ligand.data_ptr(), poses.data_ptr(), n, stride, e.data_ptr(),
                                       g.data_ptr(), gs, dw.data_ptr() if need_w else 0, nt,
                                       v_intra=v_intra, v_inter=v_inter, exact=exact, stream=_stream())
        grad_e = grad_e.to(torch.float32)
        grad_poses = None
        if ctx.needs_input_grad[0]:
            grad_poses = torch.zeros_like(poses)
            grad_poses[:, :gs] = grad_e[:, None] * g
        grad_w = (grad_e[:, None] * dw).sum(0).to(*ctx.w_like) if need_w else None
        return grad_poses, grad_w, None, None, None, None, None


def docking_energy(batch: engine.Batch, pose_ligand, poses: torch.Tensor, weights: torch.Tensor | None = None,
                   v_intra: float = 1000.0, v_inter: float = 1000.0, exact: bool = True) -> torch.Tensor:
    """Differentiable energy of `poses` ((n, >= 7 + T_max) float32 CUDA tensor)
    for the ligands `pose_ligand` of `batch`.  `weights` (n_terms,) selects the
    term weights (None: the maps' current weights, not differentiated).
    exact=True differentiates the computed energy exactly; exact=False uses the
    reference's tabulated pair derivative (what BFGS consumes)."""
    pose_ligand = torch.as_tensor(pose_ligand, device=poses.device)
    q = poses[:, 3:7]
    unit = torch.cat([poses[:, :3], q / q.norm(dim=1, keepdim=True), poses[:, 7:]], dim=1)
    return DockingEnergy.apply(unit, weights, batch, pose_ligand, float(v_intra), float(v_inter), bool(exact))
