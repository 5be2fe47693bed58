"""Sim3 pose-graph bundle adjustment, ``droid_backends.pgba``, restated in float64 numpy.

Follows HI-SLAM2 ``src/droid_kernels.cu``:
  * per-edge linearisation ``projective_transform_sim3_kernel`` (:608-858): 7-dof
    Sim3 Jacobians, the depth column taken with ``tij`` and before the self-edge
    zeroing, ``Cii`` / ``bz`` per edge;
  * the driver ``pgba_cuda`` (:1940-2044): pose blocks of the edges and of the
    caller's relative-pose factors ``Hsp`` / ``vsp`` (keys ``ii, jj, iip, jjp`` minus
    t0, negatives dropped), the Schur complement of the depths with
    ``schur_block`` at D = 7, one damped solve, ``EvT6x1_kernel`` back-substitution
    (its ``ix <= 0`` skip included) and ``disp_retr_kernel``.  Poses are not moved:
    ``dx`` is returned for the caller's Sim3 retraction.
Shared steps (keys, segmented sums, Schur, solve, back-substitution) are those of
``oracle.ba``.  Test infrastructure only (see ``oracle/__init__.py``).
"""

import numpy as np

from . import ba as _ba
from . import se3

MIN_DEPTH = _ba.MIN_DEPTH
D = 7


def validate(num_poses, ii, jj, iip, jjp, t0, t1):
    """Index preconditions under which the reference op is well defined: the BA
    edges as in ``oracle.ba.validate``; the relative-pose keys must be < t1
    (``SparseBlock::update_lhs`` :1606-1621 indexes out of range otherwise)."""
    _ba.validate(num_poses, ii, jj, t0, t1)
    iip = np.asarray(iip, dtype=np.int64)
    jjp = np.asarray(jjp, dtype=np.int64)
    if iip.shape != jjp.shape:
        raise ValueError("iip and jjp must have the same length")
    if iip.size and max(iip.max(), jjp.max()) >= t1:
        raise ValueError("iip/jjp must be < t1")


def linearize_sim3(poses, disps, intr, targets, weights, ii, jj, chunk=128):
    """``projective_transform_sim3_kernel`` (:608-858) per edge.

    Returns Hs [4,E,7,7] (Hii, Hij, Hji, Hjj as written at :836-855), vs [2,E,7],
    Eii/Eij [E,7,HW], Cii/wi [E,HW] in float64.
    """
    poses = np.asarray(poses, dtype=np.float64)
    disps = np.asarray(disps, dtype=np.float64)
    intr = np.asarray(intr, dtype=np.float64)
    targets = np.asarray(targets, dtype=np.float64)
    weights = np.asarray(weights, dtype=np.float64)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    E = ii.shape[0]
    _, ht, wd = disps.shape
    HW = ht * wd
    fx, fy = intr[0], intr[1]
    Hs = np.zeros((4, E, D, D))
    vs = np.zeros((2, E, D))
    Eii = np.zeros((E, D, HW))
    Eij = np.zeros((E, D, HW))
    Cii = np.zeros((E, HW))
    wi = np.zeros((E, HW))
    vv, uu = np.meshgrid(np.arange(ht, dtype=np.float64), np.arange(wd, dtype=np.float64), indexing="ij")
    uu = uu.reshape(-1)
    vv = vv.reshape(-1)
    for s0 in range(0, E, chunk):
        e = slice(s0, min(E, s0 + chunk))
        ie, je = ii[e], jj[e]
        tij, qij, sij = se3.rel_sim3(poses[ie, :3], poses[ie, 3:7], poses[ie, 7],
                                     poses[je, :3], poses[je, 3:7], poses[je, 7])
        tij, qij, sij = tij[:, None, :], qij[:, None, :], sij[:, None]
        Xi = se3.iproj(uu[None], vv[None], disps[ie].reshape(-1, HW), intr)
        Xj = se3.act_sim3(tij, qij, sij, Xi)
        xp, yp = se3.proj(Xj, intr)
        bad = Xj[..., 2] < MIN_DEPTH
        x, y, h = Xj[..., 0], Xj[..., 1], Xj[..., 3]
        z = np.where(bad, 0.0, Xj[..., 2])
        d = np.where(bad, 0.0, 1.0 / np.where(bad, 1.0, Xj[..., 2]))
        d2 = d * d
        w = weights[e].reshape(-1, 2, HW)
        t = targets[e].reshape(-1, 2, HW)
        wu = np.where(bad, 0.0, 0.001 * w[:, 0])
        wv = np.where(bad, 0.0, 0.001 * w[:, 1])
        ru = t[:, 0] - xp
        rv = t[:, 1] - yp
        zero = np.zeros_like(d)
        Jp = [fx * d, zero, fx * (-x * d2), zero, fy * d, fy * (-y * d2)]

        def jac(a, b, c):
            # Jj rows of one image coordinate (:733-740, :767-774): translation, rotation, scale
            return np.stack([a * h, b * h, c * h, -b * z + c * y, a * z - c * x, -a * y + b * x,
                             a * x + b * y + c * z], -1)

        Jj_u, Jj_v = jac(Jp[0], Jp[1], Jp[2]), jac(Jp[3], Jp[4], Jp[5])
        Jz_u = Jp[0] * tij[..., 0] + Jp[1] * tij[..., 1] + Jp[2] * tij[..., 2]
        Jz_v = Jp[3] * tij[..., 0] + Jp[4] * tij[..., 1] + Jp[5] * tij[..., 2]
        Cii[e] = wu * Jz_u * Jz_u + wv * Jz_v * Jz_v
        wi[e] = wu * ru * Jz_u + wv * rv * Jz_v
        selfe = (ie == je)[:, None]
        wu = np.where(selfe, 0.0, wu)
        wv = np.where(selfe, 0.0, wv)
        Ji_u = -se3.adj_sim3(tij, qij, sij, Jj_u)
        Ji_v = -se3.adj_sim3(tij, qij, sij, Jj_v)
        Jx = np.concatenate([np.concatenate([Ji_u, Jj_u], -1), np.concatenate([Ji_v, Jj_v], -1)], axis=1)
        wx = np.concatenate([wu, wv], axis=1)
        rx = np.concatenate([ru, rv], axis=1)
        H = np.matmul(np.swapaxes(Jx * wx[..., None], 1, 2), Jx)
        v = np.einsum("epn,ep->en", Jx, wx * rx)
        Hs[0, e], Hs[1, e], Hs[2, e], Hs[3, e] = H[:, :D, :D], H[:, :D, D:], H[:, D:, :D], H[:, D:, D:]
        vs[0, e], vs[1, e] = v[:, :D], v[:, D:]
        Eii[e] = np.swapaxes((wu * Jz_u)[..., None] * Ji_u + (wv * Jz_v)[..., None] * Ji_v, 1, 2)
        Eij[e] = np.swapaxes((wu * Jz_u)[..., None] * Jj_u + (wv * Jz_v)[..., None] * Jj_v, 1, 2)
    return dict(Hs=Hs, vs=vs, Eii=Eii, Eij=Eij, Cii=Cii, wi=wi)


class PGBAResult:
    """Outputs of :func:`pgba` (disps is an updated float64 copy)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def pgba(poses, disps, intrinsics, targets, weights, eta, Hsp, vsp, ii, jj, iip, jjp, t0, t1, lm, ep):
    """``pgba_cuda`` (:1940-2044) in float64 -> :class:`PGBAResult` with dx [P,7], dz
    [M,HW], disps (updated copy), ok, and the system (A, b) before damping.

    ``Hsp`` holds 4 x Np blocks 7x7 (any leading shape reshaping to [4*Np,7,7], in the
    order Hii, Hij, Hji, Hjj of the relative-pose factors), ``vsp`` 2 x Np rows of 7.
    """
    poses = np.asarray(poses, dtype=np.float64)
    disps = np.asarray(disps, dtype=np.float64).copy()
    intr = np.asarray(intrinsics, dtype=np.float64).reshape(-1)[:4]
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    iip = np.asarray(iip, dtype=np.int64)
    jjp = np.asarray(jjp, dtype=np.int64)
    validate(min(poses.shape[0], disps.shape[0]), ii, jj, iip, jjp, t0, t1)
    K, ht, wd = disps.shape
    HW = ht * wd
    P = t1 - t0
    Np = iip.shape[0]
    Hsp = np.asarray(Hsp, dtype=np.float64).reshape(4, Np, D, D)
    vsp = np.asarray(vsp, dtype=np.float64).reshape(2, Np, D)
    ts = np.arange(t0, t1, dtype=np.int64)
    kx, kk_exp, ii_exp = _ba.keys(ii, t0, t1)
    jj_exp = np.concatenate([ts, jj])
    eta = np.asarray(eta, dtype=np.float64).reshape(-1, HW)

    lin = linearize_sim3(poses, disps, intr, targets, weights, ii, jj)
    A, b = _ba.assemble_pose_system(lin["Hs"], lin["vs"], ii, jj, t0, P)
    Ap, bp = _ba.assemble_pose_system(Hsp, vsp, iip, jjp, t0, P)
    A, b = A + Ap, b + bp
    C = _ba.accum_fast(lin["Cii"], ii, kx)
    w = _ba.accum_fast(lin["wi"], ii, kx)
    Q = 1.0 / (C + eta)
    Ei = _ba.accum_fast(lin["Eii"].reshape(len(ii), D * HW), ii, ts).reshape(P, D, HW)
    E = np.concatenate([Ei, lin["Eij"]], axis=0)
    S, bS = _ba.schur_complement(E, Q, w, jj_exp, kk_exp, t0, t1)
    dx, ok = _ba.solve(A - S, b - bS, lm, ep, D=D)
    dz = _ba.back_substitute(E, Q, w, dx, ii_exp, jj_exp, kx, t0, P)
    disps.reshape(K, HW)[kx] += dz
    return PGBAResult(dx=dx, dz=dz, disps=disps, ok=ok, A=A - S, b=b - bS, kx=kx, lin=lin, Q=Q, w=w, E=E)
