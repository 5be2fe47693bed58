"""SE3 / pinhole math of the reference BA kernels, restated in float64 numpy.

Poses are ``[tx, ty, tz, qx, qy, qz, qw]`` (HI-SLAM2 ``hislam2/depth_video.py:43``,
``src/droid_kernels.cu:286-294``).  Every function broadcasts over leading axes;
the last axis holds the components.  Test infrastructure only.
"""

import numpy as np


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def act_so3(q, X):
    """Rotate X by unit quaternion q (``src/droid_kernels.cu:74-84`` actSO3)."""
    qv, qw = q[..., :3], q[..., 3:4]
    uv = 2.0 * _cross(qv, X)
    return X + qw * uv + _cross(qv, uv)


def act_se3(t, q, X):
    """Homogeneous point [X, Y, Z, d] under (t, q) (``droid_kernels.cu:86-93`` actSE3)."""
    Y = act_so3(q, X[..., :3]) + X[..., 3:4] * t
    return np.concatenate([Y, X[..., 3:4]], axis=-1)


def adj_se3(t, q, X):
    """Transposed adjoint action used for Ji = -adj(Gij, Jj) (``droid_kernels.cu:104-119``)."""
    qinv = np.concatenate([-q[..., :3], q[..., 3:4]], axis=-1)
    a, b = X[..., :3], X[..., 3:6]
    u = np.stack([t[..., 2] * a[..., 1] - t[..., 1] * a[..., 2],
                  t[..., 0] * a[..., 2] - t[..., 2] * a[..., 0],
                  t[..., 1] * a[..., 0] - t[..., 0] * a[..., 1]], axis=-1)
    return np.concatenate([act_so3(qinv, a), act_so3(qinv, b) + act_so3(qinv, u)], axis=-1)


def rel_se3(ti, qi, tj, qj):
    """Gij = Gj * Gi^-1 (``droid_kernels.cu:148-159`` relSE3)."""
    qij = np.stack([
        -qj[..., 3] * qi[..., 0] + qj[..., 0] * qi[..., 3] - qj[..., 1] * qi[..., 2] + qj[..., 2] * qi[..., 1],
        -qj[..., 3] * qi[..., 1] + qj[..., 1] * qi[..., 3] - qj[..., 2] * qi[..., 0] + qj[..., 0] * qi[..., 2],
        -qj[..., 3] * qi[..., 2] + qj[..., 2] * qi[..., 3] - qj[..., 0] * qi[..., 1] + qj[..., 1] * qi[..., 0],
        qj[..., 3] * qi[..., 3] + qj[..., 0] * qi[..., 0] + qj[..., 1] * qi[..., 1] + qj[..., 2] * qi[..., 2],
    ], axis=-1)
    tij = tj - act_so3(qij, ti)
    return tij, qij


def exp_so3(phi):
    """SO3 exponential with the reference's small-angle branch (``droid_kernels.cu:179-201``)."""
    theta_sq = np.sum(phi * phi, axis=-1)
    theta_p4 = theta_sq * theta_sq
    theta = np.sqrt(theta_sq)
    small = theta_sq < 1e-8
    safe = np.where(small, 1.0, theta)
    imag = np.where(small, 0.5 - theta_sq / 48.0 + theta_p4 / 3840.0, np.sin(0.5 * safe) / safe)
    real = np.where(small, 1.0 - theta_sq / 8.0 + theta_p4 / 384.0, np.cos(0.5 * safe))
    return np.concatenate([imag[..., None] * phi, real[..., None]], axis=-1)


def exp_se3(xi):
    """SE3 exponential, tangent order [tau, phi] (``droid_kernels.cu:216-244``)."""
    q = exp_so3(xi[..., 3:6])
    tau, phi = xi[..., :3], xi[..., 3:6]
    theta_sq = np.sum(phi * phi, axis=-1)
    theta = np.sqrt(theta_sq)
    big = theta > 1e-4
    safe_sq = np.where(big, theta_sq, 1.0)
    safe = np.where(big, theta, 1.0)
    a = np.where(big, (1.0 - np.cos(safe)) / safe_sq, 0.0)[..., None]
    b = np.where(big, (safe - np.sin(safe)) / (safe * safe_sq), 0.0)[..., None]
    c1 = _cross(phi, tau)
    c2 = _cross(phi, c1)
    t = tau + a * c1 + b * c2
    return t, q


def retr_se3(xi, t, q):
    """Left retraction exp(xi) * (t, q) (``droid_kernels.cu:1342-1360`` retrSE3)."""
    dt, dq = exp_se3(xi)
    q1 = np.stack([
        dq[..., 3] * q[..., 0] + dq[..., 0] * q[..., 3] + dq[..., 1] * q[..., 2] - dq[..., 2] * q[..., 1],
        dq[..., 3] * q[..., 1] + dq[..., 1] * q[..., 3] + dq[..., 2] * q[..., 0] - dq[..., 0] * q[..., 2],
        dq[..., 3] * q[..., 2] + dq[..., 2] * q[..., 3] + dq[..., 0] * q[..., 1] - dq[..., 1] * q[..., 0],
        dq[..., 3] * q[..., 3] - dq[..., 0] * q[..., 0] - dq[..., 1] * q[..., 1] - dq[..., 2] * q[..., 2],
    ], axis=-1)
    t1 = act_so3(dq, t) + dt
    return t1, q1


def iproj(u, v, d, intr):
    """Pixel + inverse depth -> homogeneous point (``droid_kernels.cu:66-72``)."""
    fx, fy, cx, cy = intr
    X = (u - cx) / fx
    Y = (v - cy) / fy
    one = np.ones_like(d)
    return np.stack([np.broadcast_to(X, d.shape), np.broadcast_to(Y, d.shape), one, d], axis=-1)


def proj(X, intr):
    """Pinhole projection without depth guard (``droid_kernels.cu:58-64``)."""
    fx, fy, cx, cy = intr
    with np.errstate(divide="ignore", invalid="ignore"):
        return fx * (X[..., 0] / X[..., 2]) + cx, fy * (X[..., 1] / X[..., 2]) + cy


# Sim3 poses are ``[tx, ty, tz, qx, qy, qz, qw, s]`` (``droid_kernels.cu:648-663``).

def act_sim3(t, q, s, X):
    """Homogeneous point [X, Y, Z, d] under (t, q, s): (s R X + d t, d)
    (``droid_kernels.cu:96-102`` actSim3)."""
    Y = s[..., None] * act_so3(q, X[..., :3]) + X[..., 3:4] * t
    return np.concatenate([Y, X[..., 3:4]], axis=-1)


def adj_sim3(t, q, s, X):
    """The map of ``adjSim3`` (``droid_kernels.cu:122-145``) used for Ji = -adj(Gij, Jj):
    [s R^T a, s (R^T b + R^T (a x t)) + c t, c] for X = [a, b, c] (3 + 3 + 1)."""
    Y = adj_se3(t, q, X[..., :6])
    c = X[..., 6:7]
    s_ = s[..., None]
    return np.concatenate([s_ * Y[..., :3], s_ * Y[..., 3:6] + c * t, c], axis=-1)


def rel_sim3(ti, qi, si, tj, qj, sj):
    """Gij = Gj * Gi^-1 for Sim3: qij as relSE3, sij = sj / si, tij = tj - sij R(qij) ti
    (``droid_kernels.cu:162-177`` relSim3)."""
    _, qij = rel_se3(ti, qi, tj, qj)
    sij = sj / si
    tij = tj - sij[..., None] * act_so3(qij, ti)
    return tij, qij, sij
