"""Dense bundle adjustment of ``droid_backends.ba``, restated in float64 numpy.

Follows HI-SLAM2 ``src/droid_kernels.cu``:
  * per-edge linearisation ``projective_transform_kernel`` (:364-606);
  * ``accum_cuda`` segmented sums (:1319-1339, :1413-1463);
  * ``schur_block`` + ``EEt6x6_kernel`` + ``Ev6x1_kernel`` (:1466-1560, :1689-1779);
  * ``SparseBlock::update_lhs/update_rhs/solve`` (:1598-1680);
  * ``EvT6x1_kernel`` back-substitution incl. its ``ix <= 0`` skip (:1562-1582);
  * ``pose_retr_kernel`` / ``disp_retr_kernel`` (:1363-1411);
  * the driver ``ba_cuda`` (:1820-1937).
Test infrastructure only (see ``oracle/__init__.py``).
"""

import numpy as np

from . import se3

MIN_DEPTH = 0.25  # src/droid_kernels.cu:26


def _f64(x):
    return np.asarray(x, dtype=np.float64)


def validate(num_poses, ii, jj, t0, t1):
    """Index preconditions under which the reference op is well defined.

    ``SparseBlock::update_lhs`` (:1606-1621) and ``schur_block`` (:1712-1721) index
    out of range for ii/jj >= t1, so the drop-in rejects those inputs.
    """
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    if ii.size and (ii.min() < 0 or jj.min() < 0):
        raise ValueError("ii/jj must be non-negative")
    if ii.size and (max(ii.max(), jj.max()) >= num_poses):
        raise ValueError("ii/jj index past the pose buffer")
    if ii.size and max(ii.max(), jj.max()) >= t1:
        raise ValueError("ii/jj must be < t1")
    if t0 < 0 or t1 > num_poses or t1 < t0:
        raise ValueError("need 0 <= t0 <= t1 <= num_poses")


def keys(ii, t0, t1):
    """ts, ii_exp, jj_exp handled by the caller; returns (kx, kk_exp, ii_exp).

    ``ba_cuda`` :1841-1849: ``ii_exp = cat(arange(t0,t1), ii)``,
    ``kx, kk_exp = _unique(ii_exp, sorted=True, return_inverse=True)``.
    """
    ts = np.arange(t0, t1, dtype=np.int64)
    ii_exp = np.concatenate([ts, np.asarray(ii, dtype=np.int64)])
    kx, kk_exp = np.unique(ii_exp, return_inverse=True)
    return kx.astype(np.int64), kk_exp.astype(np.int64), ii_exp


def linearize(poses, disps, intr, targets, weights, ii, jj, chunk=128):
    """Per-edge linearisation of ``projective_transform_kernel`` (:364-606).

    Returns Hs [4,E,6,6], vs [2,E,6], Eii/Eij [E,6,HW], Cii/wi [E,HW] in float64.
    Hs[0]=Hii, Hs[1]=Hij, Hs[2]=Hji, Hs[3]=Hjj as written at :586-603.
    """
    poses = _f64(poses)
    disps = _f64(disps)
    intr = _f64(intr)
    targets = _f64(targets)
    weights = _f64(weights)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    E = ii.shape[0]
    K, ht, wd = disps.shape
    HW = ht * wd
    fx, fy = intr[0], intr[1]

    Hs = np.zeros((4, E, 6, 6))
    vs = np.zeros((2, E, 6))
    Eii = np.zeros((E, 6, HW))
    Eij = np.zeros((E, 6, HW))
    Cii = np.zeros((E, HW))
    wi = np.zeros((E, HW))

    vv, uu = np.meshgrid(np.arange(ht, dtype=np.float64), np.arange(wd, dtype=np.float64), indexing="ij")
    uu = uu.reshape(-1)
    vv = vv.reshape(-1)

    for s in range(0, E, chunk):
        e = slice(s, min(E, s + chunk))
        ie, je = ii[e], jj[e]
        tij, qij = se3.rel_se3(poses[ie, :3], poses[ie, 3:], poses[je, :3], poses[je, 3:])
        tij = tij[:, None, :]
        qij = qij[:, None, :]
        d_i = disps[ie].reshape(-1, HW)
        Xi = se3.iproj(uu[None], vv[None], d_i, intr)
        Xj = se3.act_se3(tij, qij, Xi)
        xp, yp = se3.proj(Xj, intr)
        bad = Xj[..., 2] < MIN_DEPTH
        x, y, h = Xj[..., 0], Xj[..., 1], Xj[..., 3]
        z = np.where(bad, 0.0, Xj[..., 2])
        with np.errstate(divide="ignore"):
            d = np.where(bad, 0.0, 1.0 / np.where(bad, 1.0, Xj[..., 2]))
        d2 = d * d
        w = weights[e].reshape(-1, 2, HW)
        t = targets[e].reshape(-1, 2, HW)
        wu = np.where(bad, 0.0, 0.001 * w[:, 0])
        wv = np.where(bad, 0.0, 0.001 * w[:, 1])
        ru = t[:, 0] - xp
        rv = t[:, 1] - yp

        Jp = [fx * d, np.zeros_like(d), fx * (-x * d2), np.zeros_like(d), fy * d, fy * (-y * d2)]
        Jj_u = np.stack([Jp[0] * h, Jp[1] * h, Jp[2] * h,
                         -Jp[1] * z + Jp[2] * y, Jp[0] * z - Jp[2] * x, -Jp[0] * y + Jp[1] * x], -1)
        Jj_v = np.stack([Jp[3] * h, Jp[4] * h, Jp[5] * h,
                         -Jp[4] * z + Jp[5] * y, Jp[3] * z - Jp[5] * x, -Jp[3] * y + Jp[4] * x], -1)
        Jz_u = Jp[0] * tij[..., 0] + Jp[1] * tij[..., 1] + Jp[2] * tij[..., 2]
        Jz_v = Jp[3] * tij[..., 0] + Jp[4] * tij[..., 1] + Jp[5] * tij[..., 2]

        # depth terms are taken before the self-edge zeroing (:487-491, :519-523)
        Cii[e] = wu * Jz_u * Jz_u + wv * Jz_v * Jz_v
        wi[e] = wu * ru * Jz_u + wv * rv * Jz_v

        selfe = (ie == je)[:, None]
        wu = np.where(selfe, 0.0, wu)
        wv = np.where(selfe, 0.0, wv)

        Ji_u = -se3.adj_se3(tij, qij, Jj_u)
        Ji_v = -se3.adj_se3(tij, qij, Jj_v)
        Jx = np.concatenate([np.concatenate([Ji_u, Jj_u], -1), np.concatenate([Ji_v, Jj_v], -1)], axis=1)
        wx = np.concatenate([wu, wv], axis=1)
        rx = np.concatenate([ru, rv], axis=1)
        H = np.matmul(np.swapaxes(Jx * wx[..., None], 1, 2), Jx)
        v = np.einsum("epn,ep->en", Jx, wx * rx)
        Hs[0, e] = H[:, :6, :6]
        Hs[1, e] = H[:, :6, 6:]
        Hs[2, e] = H[:, 6:, :6]
        Hs[3, e] = H[:, 6:, 6:]
        vs[0, e] = v[:, :6]
        vs[1, e] = v[:, 6:]
        Eii[e] = np.swapaxes((wu * Jz_u)[..., None] * Ji_u + (wv * Jz_v)[..., None] * Ji_v, 1, 2)
        Eij[e] = np.swapaxes((wu * Jz_u)[..., None] * Jj_u + (wv * Jz_v)[..., None] * Jj_v, 1, 2)

    return dict(Hs=Hs, vs=vs, Eii=Eii, Eij=Eij, Cii=Cii, wi=wi)


def accum(data, ix, jx):
    """``accum_cuda`` (:1413-1463): out[j] = sum of data rows n with ix[n] == jx[j]."""
    data = np.asarray(data)
    out = np.zeros((len(jx),) + data.shape[1:], dtype=np.float64)
    pos = {int(k): n for n, k in enumerate(jx)}
    for n, k in enumerate(np.asarray(ix)):
        j = pos.get(int(k))
        if j is not None:
            out[j] += data[n]
    return out


def accum_fast(data, ix, jx):
    """Vectorised ``accum`` for large inputs (same result)."""
    data = np.asarray(data, dtype=np.float64)
    jx = np.asarray(jx, dtype=np.int64)
    ix = np.asarray(ix, dtype=np.int64)
    if len(jx) == 0 or len(ix) == 0:
        return np.zeros((len(jx),) + data.shape[1:], dtype=np.float64)
    order = np.argsort(jx)
    pos = np.searchsorted(jx[order], ix)
    pos = np.clip(pos, 0, len(jx) - 1)
    hit = jx[order][pos] == ix
    out = np.zeros((len(jx),) + data.shape[1:], dtype=np.float64)
    np.add.at(out, order[pos[hit]], data[hit])
    return out


def assemble_pose_system(Hs, vs, ii, jj, t0, P):
    """``update_lhs``/``update_rhs`` with keys cat(ii,ii,jj,jj)-t0 x cat(ii,jj,ii,jj)-t0.

    ``ba_cuda`` :1882-1889, ``SparseBlock`` :1598-1638: negative keys are dropped,
    duplicates are summed.
    """
    D = Hs.shape[-1]
    ii = np.asarray(ii, dtype=np.int64) - t0
    jj = np.asarray(jj, dtype=np.int64) - t0
    A = np.zeros((P, D, P, D))
    b = np.zeros((P, D))
    rows = [ii, ii, jj, jj]
    cols = [ii, jj, ii, jj]
    for blk in range(4):
        m = (rows[blk] >= 0) & (cols[blk] >= 0)
        np.add.at(A, (rows[blk][m], slice(None), cols[blk][m]), Hs[blk][m])
    for blk, keys_ in enumerate([ii, jj]):
        m = keys_ >= 0
        np.add.at(b, keys_[m], vs[blk][m])
    return A.reshape(D * P, D * P), b.reshape(-1)


def schur_rows(jj_exp, kk_exp, t0, t1):
    """Per depth slot k, the rows n of E that ``schur_block`` keeps (:1712-1721).

    graph[t] holds the rows whose pose jj_exp[n] lies in the window; rows are visited
    in increasing n.  Returns {k: [n, ...]}.
    """
    rows = {}
    for n, (j, k) in enumerate(zip(np.asarray(jj_exp), np.asarray(kk_exp))):
        if t0 <= j <= t1:
            rows.setdefault(int(k), []).append(n)
    return rows


def schur_pairs(jj_exp, kk_exp, t0, t1):
    """The (i, j, row_a, row_b, k) list of ``schur_block``'s quadruple loop (:1725-1740).

    Pure-Python loops; for small key-parity cases only.
    """
    P = t1 - t0
    graph = [[] for _ in range(P)]
    index = [[] for _ in range(P)]
    for n, (j, k) in enumerate(zip(np.asarray(jj_exp), np.asarray(kk_exp))):
        if t0 <= j <= t1:
            graph[j - t0].append(int(k))
            index[j - t0].append(n)
    out = []
    for i in range(P):
        for j in range(P):
            for a in range(len(graph[i])):
                for b in range(len(graph[j])):
                    if graph[i][a] == graph[j][b]:
                        out.append((i, j, index[i][a], index[j][b], graph[i][a]))
    return out


def schur_complement(E, Q, w, jj_exp, kk_exp, t0, t1):
    """S = sum_k sum_{a,b in rows(k)} E_a Q_k E_b^T and its rhs (``schur_block`` :1689-1779).

    Grouped by depth slot, which is the same sum as the reference's pair list.
    The rhs v[n] = sum_p Q w E[n] is taken for every row and scattered at key
    jj_exp[n]-t0, negatives dropped (``Ev6x1_kernel`` :1525-1560, :1775).
    """
    P = t1 - t0
    D, HW = E.shape[1], E.shape[-1]
    S = np.zeros((P, D, P, D))
    bS = np.zeros((P, D))
    jj_exp = np.asarray(jj_exp, dtype=np.int64)
    kk_exp = np.asarray(kk_exp, dtype=np.int64)
    for k, rows in schur_rows(jj_exp, kk_exp, t0, t1).items():
        F = E[rows].reshape(-1, HW)
        Sk = (F * Q[k]) @ F.T
        pr = jj_exp[rows] - t0
        Sk = Sk.reshape(len(rows), D, len(rows), D)
        for a in range(len(rows)):
            np.add.at(S, (pr[a], slice(None), pr), np.swapaxes(Sk[a], 0, 1))
    v = np.einsum("ndp,np->nd", E, (Q * w)[kk_exp])
    keys_ = jj_exp - t0
    m = keys_ >= 0
    np.add.at(bS, keys_[m], v[m])
    return S.reshape(D * P, D * P), bS.reshape(-1)


def solve(A, b, lm, ep, D=6):
    """``SparseBlock::solve`` (:1660-1680): diag += ep + lm*diag, LLT, zeros on failure.
    Only the lower triangle of A is read, as ``SimplicialLLT`` does."""
    n = A.shape[0]
    L = np.array(A, dtype=np.float64, copy=True)
    if n == 0:
        return np.zeros((0, D)), True
    di = np.arange(n)
    L[di, di] += ep + lm * L[di, di]
    try:
        C = np.linalg.cholesky(L)
    except np.linalg.LinAlgError:
        return np.zeros((n // D, D)), False
    y = np.linalg.solve(C, b)
    x = np.linalg.solve(C.T, y)
    return x.reshape(-1, D), True


def back_substitute(E, Q, w, dx, ii_exp, jj_exp, kx, t0, P, skip_t0=True):
    """``EvT6x1_kernel`` (:1562-1582) + ``dz = Q*(w - accum(dw, ii_exp, kx))`` (:1920).

    Rows whose pose index ix = jj_exp-t0 satisfies ix <= 0 or ix >= P get dw = 0
    (the reference skips the first window pose as well; ``skip_t0`` keeps that).
    """
    ix = np.asarray(jj_exp, dtype=np.int64) - t0
    keep = (ix > 0) if skip_t0 else (ix >= 0)
    keep &= ix < P
    dw = np.zeros((E.shape[0], E.shape[-1]))
    dw[keep] = np.einsum("ndp,nd->np", E[keep], dx[ix[keep]])
    return Q * (w - accum_fast(dw, ii_exp, kx))


class BAResult:
    """Outputs of :func:`ba` (poses/disps are updated copies, float64)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def ba(poses, disps, intrinsics, targets, weights, eta, ii, jj, t0, t1, iterations, lm, ep,
       motion_only=False, trace=False):
    """``ba_cuda`` (:1820-1937) in float64.  Returns a :class:`BAResult`.

    ``eta`` is [M or 1, H, W] (broadcast as ``C + eta.view(-1, HW)`` at :1903).
    With ``trace`` the per-iteration intermediates are kept for block-level parity.
    """
    poses = _f64(poses).copy()
    disps = _f64(disps).copy()
    intr = _f64(intrinsics)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    validate(min(poses.shape[0], disps.shape[0]), ii, jj, t0, t1)
    K, ht, wd = disps.shape
    HW = ht * wd
    P = t1 - t0
    ts = np.arange(t0, t1, dtype=np.int64)
    kx, kk_exp, ii_exp = keys(ii, t0, t1)
    jj_exp = np.concatenate([ts, jj])
    eta = _f64(eta).reshape(-1, HW)

    dx = np.zeros((P, 6))
    dz = None
    ok = True
    traces = []
    for _ in range(iterations):
        lin = linearize(poses, disps, intr, targets, weights, ii, jj)
        A, b = assemble_pose_system(lin["Hs"], lin["vs"], ii, jj, t0, P)
        it = dict(lin=lin, A=A, b=b)
        if motion_only:
            dx, ok = solve(A, b, lm, ep)
        else:
            C = accum_fast(lin["Cii"], ii, kx)
            w = accum_fast(lin["wi"], ii, kx)
            Q = 1.0 / (C + eta)
            Ei = accum_fast(lin["Eii"].reshape(len(ii), 6 * HW), ii, ts).reshape(P, 6, HW)
            E = np.concatenate([Ei, lin["Eij"]], axis=0)
            S, bS = schur_complement(E, Q, w, jj_exp, kk_exp, t0, t1)
            dx, ok = solve(A - S, b - bS, lm, ep)
            dz = back_substitute(E, Q, w, dx, ii_exp, jj_exp, kx, t0, P)
            it.update(C=C, w=w, Q=Q, E=E, S=S, bS=bS, dz=dz)
            disps.reshape(K, HW)[kx] += dz
        it.update(dx=dx, ok=ok)
        if P > 0:
            t_new, q_new = se3.retr_se3(dx, poses[t0:t1, :3], poses[t0:t1, 3:])
            poses[t0:t1, :3] = t_new
            poses[t0:t1, 3:] = q_new
        if trace:
            traces.append(it)

    return BAResult(poses=poses, disps=disps, dx=dx, dz=dz, ok=ok, kx=kx, kk_exp=kk_exp,
                    ii_exp=ii_exp, jj_exp=jj_exp, traces=traces)
