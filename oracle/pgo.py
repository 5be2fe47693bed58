"""The pose-graph terms around ``pgba`` restated in float64 numpy (TEST INFRASTRUCTURE ONLY).

* ``relative_constraints``: HI-SLAM2 ``hislam2/pgo_buffer.py:39-63``
  (``global_relative_posesim3_constraints``): per relative-pose factor the residual
  r = log(Gij Gi Gj^-1) (Gij the SE3 measurement as a Sim3 of scale 1), its Jacobians
  w.r.t. left perturbations exp(d) Gi and exp(d) Gj, and Hsp = pw [Ji' W Ji, Ji' W Jj,
  Jj' W Ji, Jj' W Jj], vsp = -pw [Ji' W r, Jj' W r], chi2 = sum r'r, chi2_scaled =
  sum r' W r.
* ``retract``: ``geom/ba.py:27-29`` ``pose_retr`` on Sim3 poses, G <- exp(dx) G for the
  poses of [t0, t1) (``hislam2/depth_video.py:267``).

The reference computes the group operations with lietorch, which is not installed here
(a third-party submodule of HI-SLAM2, princeton-vl/lietorch, unpinned).  This module does
not restate lietorch's code: it uses the definitions its Sim3 follows -- elements
X -> s R X + t stored as [t, q (x y z w), s], tangent [tau, phi, sigma] with the algebra
element [[sigma I + [phi]x, tau], [0, 0]] -- and evaluates exp and log as scipy's matrix
exponential and principal matrix logarithm of the 4x4 forms.  The reference's Jacobians
are central differences with step 1e-8; here the derivative is taken with a five-point
stencil of step 1e-4 on the same function (truncation ~1e-16, rounding ~1e-11), i.e. the
quantity the reference's differences approximate.  The group conventions are pinned by
identities in ``tests/test_oracle_pgo.py`` (exp/log inverse pairs, Ji = Ad(Gij) and
Jj = -I at a zero residual), and the procedure around them by the reference's own
``num_jacobi`` / ``global_relative_posesim3_constraints`` run on a Sim3 stand-in
(``tests/golden/make_golden_pgo.py``); against lietorch itself the parity is unpinned.
"""

import numpy as np
from scipy.linalg import expm, logm


def quat_to_rot(q):
    x, y, z, w = np.asarray(q, np.float64) / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def rot_to_quat(R):
    """Unit quaternion (x y z w, w >= 0) of a rotation matrix by Shepperd's method: the
    largest of 4w^2, 4x^2, 4y^2, 4z^2 from the diagonal, the others from off-diagonal sums
    divided by it, so small components keep full relative accuracy."""
    tr = R[0, 0] + R[1, 1] + R[2, 2]
    k = int(np.argmax([tr, R[0, 0], R[1, 1], R[2, 2]]))
    if k == 0:
        w = np.sqrt(1 + tr) / 2
        q = [(R[2, 1] - R[1, 2]) / (4 * w), (R[0, 2] - R[2, 0]) / (4 * w), (R[1, 0] - R[0, 1]) / (4 * w), w]
    elif k == 1:
        x = np.sqrt(1 + 2 * R[0, 0] - tr) / 2
        q = [x, (R[0, 1] + R[1, 0]) / (4 * x), (R[0, 2] + R[2, 0]) / (4 * x), (R[2, 1] - R[1, 2]) / (4 * x)]
    elif k == 2:
        y = np.sqrt(1 + 2 * R[1, 1] - tr) / 2
        q = [(R[0, 1] + R[1, 0]) / (4 * y), y, (R[1, 2] + R[2, 1]) / (4 * y), (R[0, 2] - R[2, 0]) / (4 * y)]
    else:
        z = np.sqrt(1 + 2 * R[2, 2] - tr) / 2
        q = [(R[0, 2] + R[2, 0]) / (4 * z), (R[1, 2] + R[2, 1]) / (4 * z), z, (R[1, 0] - R[0, 1]) / (4 * z)]
    q = np.array(q)
    return -q if q[3] < 0 else q


def to_matrix(p):
    """[t, q, s] (or [t, q] with s = 1) -> 4x4 [[s R, t], [0, 1]]."""
    p = np.asarray(p, np.float64)
    s = p[7] if p.shape[0] == 8 else 1.0
    M = np.eye(4)
    M[:3, :3] = s * quat_to_rot(p[3:7])
    M[:3, 3] = p[:3]
    return M


def from_matrix(M):
    s = np.cbrt(np.linalg.det(M[:3, :3]))
    return np.concatenate([M[:3, 3], rot_to_quat(M[:3, :3] / s), [s]])


def hat(xi):
    tau, phi, sigma = xi[:3], xi[3:6], xi[6]
    A = np.zeros((4, 4))
    A[:3, :3] = sigma * np.eye(3) + np.array([[0, -phi[2], phi[1]], [phi[2], 0, -phi[0]], [-phi[1], phi[0], 0]])
    A[:3, 3] = tau
    return A


def exp(xi):
    return expm(hat(np.asarray(xi, np.float64)))


def log(M):
    A = np.real(logm(M))
    sigma = np.trace(A[:3, :3]) / 3
    K = A[:3, :3] - sigma * np.eye(3)
    return np.array([A[0, 3], A[1, 3], A[2, 3], K[2, 1], K[0, 2], K[1, 0], sigma])


def adjoint(M):
    """Ad of a Sim3 element: exp(Ad xi) = G exp(xi) G^-1, tangent order [tau, phi, sigma]."""
    sR, t = M[:3, :3], M[:3, 3]
    s = np.cbrt(np.linalg.det(sR))
    R = sR / s
    tx = np.array([[0, -t[2], t[1]], [t[2], 0, -t[0]], [-t[1], t[0], 0]])
    Ad = np.zeros((7, 7))
    Ad[:3, :3] = sR
    Ad[:3, 3:6] = tx @ R
    Ad[:3, 6] = -t
    Ad[3:6, 3:6] = R
    Ad[6, 6] = 1.0
    return Ad


def _residual(Gij, Gi, Gj):
    return log(Gij @ Gi @ np.linalg.inv(Gj))


def _jacobian(f, h=1e-4):
    cols = []
    for k in range(7):
        d = np.zeros(7)
        d[k] = h
        cols.append((8 * (f(d) - f(-d)) - (f(2 * d) - f(-2 * d))) / (12 * h))
    return np.stack(cols, -1)


def factor_terms(pi, pj, rel):
    """(r [7], Ji [7,7], Jj [7,7]) of one factor; pi, pj Sim3 [8], rel SE3 [7]."""
    Gi, Gj, Gij = to_matrix(pi), to_matrix(pj), to_matrix(rel)
    r = _residual(Gij, Gi, Gj)
    Ji = _jacobian(lambda d: _residual(Gij, exp(d) @ Gi, Gj))
    Jj = _jacobian(lambda d: _residual(Gij, Gi, exp(d) @ Gj))
    return r, Ji, Jj


def relative_constraints(ii, jj, poses, rel_poses, infos, pw=1e-5):
    """poses [N, 8], rel_poses [Np, 7], infos [Np, 7, 7] -> (Hsp [4, Np, 7, 7], vsp [2, Np, 7],
    chi2, chi2_scaled, r [Np, 7], Ji, Jj [Np, 7, 7])."""
    poses = np.asarray(poses, np.float64)
    rel_poses = np.asarray(rel_poses, np.float64)
    infos = np.asarray(infos, np.float64)
    Np = len(ii)
    r = np.zeros((Np, 7))
    Ji = np.zeros((Np, 7, 7))
    Jj = np.zeros((Np, 7, 7))
    for n in range(Np):
        r[n], Ji[n], Jj[n] = factor_terms(poses[ii[n]], poses[jj[n]], rel_poses[n])
    wJiT = pw * np.transpose(Ji, (0, 2, 1)) @ infos
    wJjT = pw * np.transpose(Jj, (0, 2, 1)) @ infos
    Hsp = np.stack([wJiT @ Ji, wJiT @ Jj, wJjT @ Ji, wJjT @ Jj])
    vsp = -np.stack([wJiT @ r[..., None], wJjT @ r[..., None]])[..., 0]
    chi2 = float((r * r).sum())
    chi2_scaled = float(np.einsum("na,nab,nb->", r, infos, r))
    return Hsp, vsp, chi2, chi2_scaled, r, Ji, Jj


def retract(poses, dx, t0, t1):
    """poses [N, 8] Sim3 -> a copy with poses[t0 + k] = exp(dx[k]) poses[t0 + k]."""
    out = np.array(poses, np.float64)
    for k in range(t1 - t0):
        out[t0 + k] = from_matrix(exp(np.asarray(dx[k], np.float64)) @ to_matrix(out[t0 + k]))
    return out
