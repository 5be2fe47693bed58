"""HI-SLAM2's pure-PyTorch bundle adjustment, restated (TEST / BASELINE INFRASTRUCTURE ONLY).

The reference's Python path -- ``hislam2/geom/ba.py:BA`` (:32-108) with
``hislam2/geom/chol.py:schur_solve`` (:47-78) and
``hislam2/geom/projective_ops.py:projective_transform`` (:42-88) -- cannot be
imported here: it needs ``lietorch`` (SE3 group) and ``torch_scatter``, neither of
which is installed.  This module restates it with a self-written quaternion SE3
and ``index_add_`` in place of ``scatter_sum``, keeping its numerics: MIN_DEPTH
0.2 on both depths, the 0.001 weight scale, damping of the pose Hessian before
the Schur complement (``H + (ep + lm H) I``), ``C + eta + 1e-7``, a dense E of
shape [P, M, 6, HW], the dzcov term, and the final ``disps > 10 -> 0`` and
``clamp(min=0.001)``.  It is the CPU baseline that bench.py times on the host
cores; it differs from the CUDA operator (``droid_backends.ba``) in exactly the
ways listed above, so it is never used as a parity oracle.

Poses are [N, 7] (t, q xyzw) like the CUDA operator's; the fixed poses are the
first ``t0`` (``fixedp`` in the reference).
"""

import torch

MIN_DEPTH = 0.2  # hislam2/geom/projective_ops.py:6


def _cross(a, b):
    return torch.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                        a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                        a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def quat_rotate(q, X):
    uv = 2.0 * _cross(q[..., :3], X)
    return X + q[..., 3:4] * uv + _cross(q[..., :3], uv)


def quat_mul(a, b):
    return torch.cat([a[..., 3:4] * b[..., :3] + b[..., 3:4] * a[..., :3] + _cross(a[..., :3], b[..., :3]),
                      a[..., 3:4] * b[..., 3:4] - (a[..., :3] * b[..., :3]).sum(-1, keepdim=True)], -1)


def quat_to_matrix(q):
    x, y, z, w = q.unbind(-1)
    return torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1).view(
        *q.shape[:-1], 3, 3)


def relative(pi, pj):
    """Gij = Gj * Gi^-1 for poses [.., 7] -> (t [.., 3], q [.., 4])."""
    qi_inv = torch.cat([-pi[..., 3:6], pi[..., 6:7]], -1)
    q = quat_mul(pj[..., 3:], qi_inv)
    t = pj[..., :3] - quat_rotate(q, pi[..., :3])
    return t, q


def se3_exp(xi):
    """Tangent [tau, phi] -> (t, q); the left retraction ``poses.retr(dx)`` of lietorch."""
    tau, phi = xi[..., :3], xi[..., 3:]
    th2 = (phi * phi).sum(-1, keepdim=True)
    th = th2.sqrt()
    small = th2 < 1e-8
    ths = torch.where(small, torch.ones_like(th), th)
    imag = torch.where(small, 0.5 - th2 / 48.0, torch.sin(0.5 * ths) / ths)
    q = torch.cat([imag * phi, torch.cos(0.5 * th)], -1)
    a = torch.where(small, 0.5 - th2 / 24.0, (1 - torch.cos(ths)) / ths ** 2)
    b = torch.where(small, 1.0 / 6.0 - th2 / 120.0, (ths - torch.sin(ths)) / ths ** 3)
    c1 = _cross(phi, tau)
    t = tau + a * c1 + b * _cross(phi, c1)
    return t, q


def retr(poses, dx):
    t, q = se3_exp(dx)
    return torch.cat([quat_rotate(q, poses[..., :3]) + t, quat_mul(q, poses[..., 3:])], -1)


def projective_transform(poses, disps, intrinsics, ii, jj):
    """``projective_transform(..., jacobian=True)`` for one batch: coords [E,H,W,2],
    valid [E,H,W,1], Ji/Jj [E,H,W,2,6], Jz [E,H,W,2,1]."""
    ht, wd = disps.shape[-2:]
    fx, fy, cx, cy = intrinsics.unbind(-1)
    y, x = torch.meshgrid(torch.arange(ht, dtype=disps.dtype), torch.arange(wd, dtype=disps.dtype), indexing="ij")
    d = disps[ii]
    X0 = torch.stack([(x - cx) / fx, (y - cy) / fy, torch.ones_like(x)], -1).expand(len(ii), ht, wd, 3)
    t, q = relative(poses[ii], poses[jj])
    R = quat_to_matrix(q)
    X = torch.einsum("eab,ehwb->ehwa", R, X0) + d[..., None] * t[:, None, None, :]
    Xx, Xy, Z = X.unbind(-1)
    coords = torch.stack([fx * Xx / Z + cx, fy * Xy / Z + cy], -1)
    valid = ((Z > MIN_DEPTH) & (X0[..., 2] > MIN_DEPTH)).to(disps.dtype)[..., None]
    o = torch.zeros_like(d)
    # action Jacobian of the homogeneous point [X, Y, Z, d] (projective_ops.py:18-31)
    Ja = torch.stack([d, o, o, o, Z, -Xy,
                      o, d, o, -Z, o, Xx,
                      o, o, d, Xy, -Xx, o], -1).view(*d.shape, 3, 6)
    iz = 1.0 / Z
    Jp = torch.stack([fx * iz, o, -fx * Xx * iz * iz,
                      o, fy * iz, -fy * Xy * iz * iz], -1).view(*d.shape, 2, 3)
    Jj = Jp @ Ja
    # Ji = -Jj Adj(Gij): Adj = [[R, [t]x R], [0, R]]
    tx = torch.zeros(len(ii), 3, 3, dtype=disps.dtype)
    tx[:, 0, 1], tx[:, 0, 2], tx[:, 1, 2] = -t[:, 2], t[:, 1], -t[:, 0]
    tx[:, 1, 0], tx[:, 2, 0], tx[:, 2, 1] = t[:, 2], -t[:, 1], t[:, 0]
    adj = torch.zeros(len(ii), 6, 6, dtype=disps.dtype)
    adj[:, :3, :3] = R
    adj[:, :3, 3:] = tx @ R
    adj[:, 3:, 3:] = R
    Ji = -torch.einsum("ehwab,ebc->ehwac", Jj, adj)
    Jz = (Jp @ t[:, None, None, :, None])          # d X / d disp = t
    return coords, valid, (Ji, Jj, Jz)


def _scatter_mat(A, ii, jj, n, m):
    """``safe_scatter_add_mat`` (geom/ba.py:13-15): A [N, ...] summed into [n*m, ...]."""
    v = (ii >= 0) & (jj >= 0) & (ii < n) & (jj < m)
    out = torch.zeros(n * m, *A.shape[1:], dtype=A.dtype)
    return out.index_add_(0, ii[v] * m + jj[v], A[v])


def _scatter_vec(b, ii, n):
    v = (ii >= 0) & (ii < n)
    out = torch.zeros(n, *b.shape[1:], dtype=b.dtype)
    return out.index_add_(0, ii[v], b[v])


def schur_solve(H, E, C, v, w, ep, lm):
    """``geom/chol.py:schur_solve`` (:47-78) for one batch; returns dx [P,6], dz [M,HW], dzcov [M,HW]."""
    P, M, D, HW = E.shape
    H = H.permute(0, 2, 1, 3).reshape(P * D, P * D)
    E = E.permute(0, 2, 1, 3).reshape(P * D, M * HW)
    Q = (1.0 / C).view(M * HW, 1)
    H = H + (ep + lm * H) * torch.eye(P * D, dtype=H.dtype)
    v = v.reshape(P * D, 1)
    w = w.reshape(M * HW, 1)
    Et = E.t()
    S = H - E @ (Q * Et)
    v = v - E @ (Q * w)
    try:
        L = torch.linalg.cholesky(S)
        dx = torch.cholesky_solve(v, L)
    except RuntimeError:            # CholeskySolver (chol.py:8-22): zero update on failure
        L = torch.zeros_like(S)
        dx = torch.zeros_like(v)
    dz = Q * (w - Et @ dx)
    F = torch.linalg.solve_triangular(L, E * Q[:, 0], upper=False) if bool(L.any()) else torch.zeros_like(E)
    dzcov = (F * F).sum(0) + Q[:, 0]
    return dx.reshape(P, D), dz.reshape(M, HW), dzcov.reshape(M, HW)


def BA(target, weight, eta, poses, disps, intrinsics, ii, jj, t0, ep=0.1, lm=1e-4):
    """One iteration of ``geom/ba.py:BA`` (:32-108).  target/weight [E, H, W, 2],
    eta [M, H, W], poses [N, 7], disps [N, H, W], intrinsics [4]; the first t0 poses
    are fixed.  Returns (poses, disps, dzcov)."""
    N, ht, wd = disps.shape
    HW = ht * wd
    E = len(ii)
    D = 6
    coords, valid, (Ji, Jj, Jz) = projective_transform(poses, disps, intrinsics, ii, jj)
    r = (target - coords).reshape(E, HW * 2, 1)
    w = 0.001 * (valid * weight).reshape(E, HW * 2, 1)
    Ji = Ji.reshape(E, HW * 2, D)
    Jj = Jj.reshape(E, HW * 2, D)
    wJiT = (w * Ji).transpose(1, 2)
    wJjT = (w * Jj).transpose(1, 2)
    Jz = Jz.reshape(E, HW, 2)
    Hii, Hij, Hji, Hjj = wJiT @ Ji, wJiT @ Jj, wJjT @ Ji, wJjT @ Jj
    vi, vj = (wJiT @ r)[..., 0], (wJjT @ r)[..., 0]
    Ei = (wJiT.view(E, D, HW, 2) * Jz[:, None]).sum(-1)
    Ej = (wJjT.view(E, D, HW, 2) * Jz[:, None]).sum(-1)
    w = w.view(E, HW, 2)
    r = r.view(E, HW, 2)
    wk = (w * r * Jz).sum(-1)
    Ck = (w * Jz * Jz).sum(-1)
    kx, kk = torch.unique(ii, return_inverse=True)
    M = len(kx)
    P = N - t0
    ii0, jj0 = ii - t0, jj - t0
    H = (_scatter_mat(Hii, ii0, ii0, P, P) + _scatter_mat(Hij, ii0, jj0, P, P) +
         _scatter_mat(Hji, jj0, ii0, P, P) + _scatter_mat(Hjj, jj0, jj0, P, P))
    Emat = _scatter_mat(Ei, ii0, kk, P, M) + _scatter_mat(Ej, jj0, kk, P, M)
    v = _scatter_vec(vi, ii0, P) + _scatter_vec(vj, jj0, P)
    C = _scatter_vec(Ck, kk, M)
    wv = _scatter_vec(wk, kk, M)
    C = C + eta.reshape(M, HW) + 1e-7
    dx, dz, dzcov = schur_solve(H.view(P, P, D, D), Emat.view(P, M, D, HW), C, v, wv, ep, lm)
    poses = poses.clone()
    poses[t0:] = retr(poses[t0:], dx)
    disps = disps.clone()
    disps.view(N, HW).index_add_(0, kx, dz)
    disps = torch.where(disps > 10, torch.zeros_like(disps), disps).clamp(min=0.001)
    return poses, disps, dzcov
