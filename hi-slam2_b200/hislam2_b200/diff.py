"""Differentiable bundle-adjustment step on the B200 kernels.

:class:`BAStep` is a ``torch.autograd.Function`` around ONE Levenberg-Marquardt
iteration of ``droid_backends.ba`` (motion_only = False): forward returns the
step's pose update dx [t1-t0, 6] and disparity update dz [M, H*W] (the caller
retracts them, as ``ba`` does in place); backward returns the gradients with
respect to targets, weights and eta from the hand-written adjoint kernels
(``hs2_ba_adjoint``: implicit differentiation through the damped Schur solve,
reusing the forward's system build and Cholesky).  The linearisation point --
poses, disparities, intrinsics and the edge list -- is not differentiated.

The reference differentiates its BA only through the pure-PyTorch path
(``hislam2/geom/ba.py``, ``hislam2/geom/chol.py:8-22`` ``CholeskySolver``); its
CUDA ``ba`` has no backward.
"""

import torch

from . import backends


class BAStep(torch.autograd.Function):

    @staticmethod
    def forward(ctx, targets, weights, eta, poses, disps, intrinsics, ii, jj, t0, t1, lm, ep):
        p, d = poses.detach().clone(), disps.detach().clone()
        dx, dz, _ = backends.ba(p, d, intrinsics, targets.detach(), weights.detach(), eta.detach(), ii, jj, t0, t1,
                                1, lm, ep, False)
        ctx.save_for_backward(targets, weights, eta, poses, disps, intrinsics, ii, jj, dx)
        ctx.args = (t0, t1, lm, ep)
        return dx, dz

    @staticmethod
    def backward(ctx, grad_dx, grad_dz):
        targets, weights, eta, poses, disps, intrinsics, ii, jj, dx = ctx.saved_tensors
        t0, t1, lm, ep = ctx.args
        if grad_dx is None:
            grad_dx = torch.zeros_like(dx)
        if grad_dz is None:
            raise RuntimeError("BAStep.backward: dz's gradient is required (use zeros)")
        gt, gw, ge, _ = backends.ba_adjoint(poses, disps, intrinsics, targets.detach(), weights.detach(),
                                            eta.detach(), ii, jj, t0, t1, lm, ep, dx, grad_dx.float(),
                                            grad_dz.float())
        return gt, gw, ge, None, None, None, None, None, None, None, None, None


def ba_step(targets, weights, eta, poses, disps, intrinsics, ii, jj, t0, t1, lm=1e-4, ep=0.1):
    """(dx, dz) of one differentiable LM step; see :class:`BAStep`."""
    return BAStep.apply(targets, weights, eta, poses, disps, intrinsics, ii, jj, t0, t1, lm, ep)
