"""Seeded synthetic BA / correlation problems with HI-SLAM2's runtime shapes.

No dataset is needed: poses, disparities, flow targets, confidences and
feature maps are drawn from fixed distributions with a seeded generator, at the
shapes HI-SLAM2 uses (1/8-resolution grids, 128-d features, 4 pyramid levels).

Workloads (name: keyframes, grid, edges, window, iterations, damping):
  * ``frontend_small``  8 kf, 48x64 (384x512 image), 24 edges i->i+k (k=1..3, folded
    back to i-k at the end of the clip), t0=2, 2 iters, lm=1e-4, ep=0.1, radius 3,
    disps U[0.2,1.0];
  * ``frontend``        25 kf, 43x77 (344x616 image), 258 edges: all 1<=|i-j|<=3
    (138) + 60 random long pairs in both directions (120), t0=2, 4 iters,
    lm=1e-4, ep=0.1, radius 4, disps U[0.1,2.0];
  * ``backend300``      300 kf, 43x77, 6000 edges: all 1<=|i-j|<=2 (1194) + 2403
    random loop pairs |i-j|>2 in both directions (4806), t0=10, 8 iters,
    lm=1e-5, ep=1e-2, 5% target outliers U[-20,20] px with weight 0;
  * ``clips2x7``        2 clips x 7 frames, 48x64, all 42 edges i!=j per clip, radius 4;
  * ``tiny6`` / ``tiny7`` 6 / 7 kf at 12x16 (96x128 image), 3 iters: the golden-fixture
    problems (a self-edge, a duplicate edge, a loop pair; tiny7 optimises the window
    [1, 6) of a 7-frame buffer whose last frame is unused, with 5% outliers).
Common: ground-truth poses = identity (+) se3 noise sigma 0.05, targets = ground-
truth reprojection + N(0, 0.5 px), weights U[0,1] per channel, eta = 1e-3; the
optimised poses start from the ground truth (+) se3 noise sigma 0.01.
Intrinsics: Replica's 600/600/599.5/339.5 on 1200x680, resized to the image and
divided by 8.
"""

import math

import torch

CONFIGS = {
    "frontend_small": dict(K=8, ht=48, wd=64, img=(384, 512), t0=2, iters=2, lm=1e-4, ep=0.1, radius=3,
                           disp=(0.2, 1.0), outliers=0.0),
    "frontend": dict(K=25, ht=43, wd=77, img=(344, 616), t0=2, iters=4, lm=1e-4, ep=0.1, radius=4,
                     disp=(0.1, 2.0), outliers=0.0),
    "backend300": dict(K=300, ht=43, wd=77, img=(344, 616), t0=10, iters=8, lm=1e-5, ep=1e-2, radius=4,
                       disp=(0.1, 2.0), outliers=0.05),
    "clips2x7": dict(K=7, ht=48, wd=64, img=(384, 512), t0=2, iters=2, lm=1e-4, ep=0.1, radius=4,
                     disp=(0.2, 1.0), outliers=0.0),
    "tiny6": dict(K=6, ht=12, wd=16, img=(96, 128), t0=2, iters=3, lm=1e-4, ep=0.1, radius=3,
                  disp=(0.2, 1.0), outliers=0.0),
    "tiny7": dict(K=7, ht=12, wd=16, img=(96, 128), t0=1, t1=6, iters=3, lm=1e-4, ep=0.1, radius=3,
                  disp=(0.2, 1.0), outliers=0.05),
}


def intrinsics_for(img_hw):
    """Replica pinhole (fx, fy, cx, cy) = (600, 600, 599.5, 339.5) at 1200x680, resized and /8."""
    h, w = img_hw
    sx, sy = w / 1200.0, h / 680.0
    return torch.tensor([600.0 * sx / 8, 600.0 * sy / 8, 599.5 * sx / 8, 339.5 * sy / 8], dtype=torch.float64)


# ------------------------------------------------------------- SE3 in torch
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


def se3_exp(xi):
    """Tangent [tau, phi] -> pose [t, q(xyzw)] (float64)."""
    tau, phi = xi[..., :3], xi[..., 3:]
    th = phi.norm(dim=-1, keepdim=True).clamp_min(1e-12)
    q = torch.cat([torch.sin(0.5 * th) / th * phi, torch.cos(0.5 * th)], -1)
    a = (1 - torch.cos(th)) / th ** 2
    b = (th - torch.sin(th)) / th ** 3
    c1 = _cross(phi, tau)
    t = tau + a * c1 + b * _cross(phi, c1)
    return torch.cat([t, q], -1)


def pose_compose(a, b):
    """a * b for poses [t, q]."""
    return torch.cat([quat_rotate(a[..., 3:], b[..., :3]) + a[..., :3], quat_mul(a[..., 3:], b[..., 3:])], -1)


def reproject(poses, disps, intr, ii, jj):
    """Pixel grid of frame ii mapped into frame jj: coords [E, H, W, 2] (float64)."""
    poses = poses.double()
    disps = disps.double()
    intr = intr.double()
    K, ht, wd = disps.shape
    fx, fy, cx, cy = intr.tolist()
    v, u = torch.meshgrid(torch.arange(ht, dtype=torch.float64), torch.arange(wd, dtype=torch.float64),
                          indexing="ij")
    pi, pj = poses[ii], poses[jj]
    qi_inv = torch.cat([-pi[:, 3:6], pi[:, 6:7]], -1)
    qij = quat_mul(pj[:, 3:], qi_inv)
    tij = pj[:, :3] - quat_rotate(qij, pi[:, :3])
    X = torch.stack([(u - cx) / fx, (v - cy) / fy, torch.ones_like(u)], -1)[None].expand(len(ii), ht, wd, 3)
    d = disps[ii][..., None]
    Y = quat_rotate(qij[:, None, None], X) + d * tij[:, None, None]
    z = Y[..., 2]
    return torch.stack([fx * Y[..., 0] / z + cx, fy * Y[..., 1] / z + cy], -1)


# ------------------------------------------------------------------ edges
def edges_for(name, K, g):
    if name == "frontend_small":
        e = []
        for i in range(K):
            for k in (1, 2, 3):
                j = i + k if i + k < K else i - k
                e.append((i, j))
        return e
    if name in ("frontend", "backend300"):
        rad = 3 if name == "frontend" else 2
        npairs = 60 if name == "frontend" else 2403
        e = [(i, j) for i in range(K) for j in range(K) if i != j and abs(i - j) <= rad]
        seen = set()
        while len(seen) < npairs:
            i, j = torch.randint(0, K, (2,), generator=g).tolist()
            if abs(i - j) > rad and (min(i, j), max(i, j)) not in seen:
                seen.add((min(i, j), max(i, j)))
        for i, j in sorted(seen):
            e.append((i, j))
            e.append((j, i))
        return e
    if name == "clips2x7":
        return [(i, j) for i in range(K) for j in range(K) if i != j]
    if name == "tiny6":
        # all 1<=|i-j|<=2, a loop pair, a duplicate edge and a self-edge
        e = [(i, j) for i in range(K) for j in range(K) if i != j and abs(i - j) <= 2]
        return e + [(0, 5), (5, 0), (3, 4), (2, 2)]
    if name == "tiny7":
        # window [1, 6) of a 7-frame buffer; frame 6 takes no part (edges need ii, jj < t1)
        e = [(i, j) for i in range(6) for j in range(6) if i != j and abs(i - j) <= 2]
        return e + [(0, 3), (5, 1)]
    raise KeyError(name)


def make_ba_problem(name="frontend_small", seed=0, device="cpu"):
    """Inputs of ``droid_backends.ba`` for workload ``name`` (see module docstring).

    Returns a dict with poses [K,7], disps [K,H,W], intrinsics [4], targets and
    weights [E,2,H,W], eta [K,H,W], ii/jj [E] (int64), t0, t1, iters, lm, ep, radius,
    and the ground truth poses_gt / disps_gt.
    """
    cfg = CONFIGS[name]
    g = torch.Generator().manual_seed(seed)
    K, ht, wd = cfg["K"], cfg["ht"], cfg["wd"]
    intr = intrinsics_for(cfg["img"])
    xi = 0.05 * torch.randn(K, 6, generator=g, dtype=torch.float64)
    poses_gt = se3_exp(xi)
    lo, hi = cfg["disp"]
    disps_gt = lo + (hi - lo) * torch.rand(K, ht, wd, generator=g, dtype=torch.float64)
    e = edges_for(name, K, g)
    ii = torch.tensor([a for a, _ in e], dtype=torch.int64)
    jj = torch.tensor([b for _, b in e], dtype=torch.int64)
    E = len(e)
    coords = reproject(poses_gt, disps_gt, intr, ii, jj)               # [E,H,W,2]
    targets = coords + 0.5 * torch.randn(coords.shape, generator=g, dtype=torch.float64)
    weights = torch.rand(E, ht, wd, 2, generator=g, dtype=torch.float64)
    if cfg["outliers"] > 0:
        out = torch.rand(E, ht, wd, generator=g) < cfg["outliers"]
        noise = -20 + 40 * torch.rand(E, ht, wd, 2, generator=g, dtype=torch.float64)
        targets = torch.where(out[..., None], targets + noise, targets)
        weights = torch.where(out[..., None], torch.zeros_like(weights), weights)
    t0, t1 = cfg["t0"], cfg.get("t1", K)
    poses = poses_gt.clone()
    pert = se3_exp(0.01 * torch.randn(K, 6, generator=g, dtype=torch.float64))
    poses[t0:t1] = pose_compose(pert[t0:t1], poses_gt[t0:t1])
    f32 = dict(dtype=torch.float32, device=device)
    return dict(
        poses=poses.to(**f32).contiguous(),
        disps=disps_gt.to(**f32).contiguous(),
        intrinsics=intr.to(**f32),
        targets=targets.permute(0, 3, 1, 2).to(**f32).contiguous(),
        weights=weights.permute(0, 3, 1, 2).to(**f32).contiguous(),
        eta=torch.full((K, ht, wd), 1e-3, **f32),
        ii=ii.to(device), jj=jj.to(device),
        t0=t0, t1=t1, iters=cfg["iters"], lm=cfg["lm"], ep=cfg["ep"], radius=cfg["radius"],
        poses_gt=poses_gt.to(**f32), disps_gt=disps_gt.to(**f32),
    )


def make_corr_problem(name="frontend", seed=0, device="cpu", num_edges=None, dtype=torch.float16,
                      num_levels=4):
    """Feature maps [K,128,H,W] ~ N(0,1)/sqrt(128) and lookup coordinates for the edges of
    workload ``name`` (optionally the first ``num_edges``).

    Returns fmaps, ii, jj, coords [E,H,W,2] (ground-truth reprojection + N(0,1) px),
    radius and num_levels.
    """
    cfg = CONFIGS[name]
    g = torch.Generator().manual_seed(seed + 1000)
    p = make_ba_problem(name, seed)
    K, ht, wd = cfg["K"], cfg["ht"], cfg["wd"]
    fmaps = torch.randn(K, 128, ht, wd, generator=g) / math.sqrt(128.0)
    ii, jj = p["ii"], p["jj"]
    if num_edges is not None:
        ii, jj = ii[:num_edges], jj[:num_edges]
    coords = reproject(p["poses_gt"], p["disps_gt"], p["intrinsics"], ii, jj)
    coords = coords + torch.randn(coords.shape, generator=g, dtype=torch.float64)
    return dict(fmaps=fmaps.to(device=device, dtype=dtype), ii=ii.to(device), jj=jj.to(device),
                coords=coords.to(device=device, dtype=torch.float32), radius=cfg["radius"],
                num_levels=num_levels)


def make_pgba_problem(name="frontend_small", seed=0, device="cpu", num_factors=None, scale_sigma=0.05,
                      info_range=(3.0, 6.0)):
    """Inputs of ``droid_backends.pgba`` for workload ``name``: the BA problem of the same
    name with Sim3 poses [K, 8] (scale exp(N(0, scale_sigma)) appended) and
    ``num_factors`` (default 2K) relative-pose factors between random frames below t1,
    about a quarter of them touching frames before t0.  Each factor has Jacobians
    Ji, Jj ~ N(0, 1) (7x7), information diag(10^U(info_range)), weight pw = 1e-3 and
    residual r ~ N(0, 0.01): Hsp = pw [Ji' W Ji, Ji' W Jj, Jj' W Ji, Jj' W Jj]
    [4, 1, Np, 7, 7] and vsp = -pw [Ji' W r, Jj' W r] [2, 1, Np, 7], the layout of
    ``hislam2/pgo_buffer.py:global_relative_posesim3_constraints``.
    """
    p = make_ba_problem(name, seed=seed, device="cpu")
    g = torch.Generator().manual_seed(seed + 2000)
    K, t0, t1 = p["poses"].shape[0], p["t0"], p["t1"]
    s = torch.exp(scale_sigma * torch.randn(K, 1, generator=g, dtype=torch.float64)).float()
    poses = torch.cat([p["poses"], s], 1)
    Np = 2 * K if num_factors is None else num_factors
    iip = torch.randint(0, t1, (Np,), generator=g)
    jjp = torch.randint(max(t0, 1), t1, (Np,), generator=g) if t1 > max(t0, 1) else torch.zeros(Np, dtype=torch.long)
    Ji = torch.randn(Np, 7, 7, generator=g, dtype=torch.float64)
    Jj = torch.randn(Np, 7, 7, generator=g, dtype=torch.float64)
    lo, hi = info_range
    W = torch.diag_embed(10.0 ** (lo + (hi - lo) * torch.rand(Np, 7, generator=g, dtype=torch.float64)))
    r = 0.01 * torch.randn(Np, 7, 1, generator=g, dtype=torch.float64)
    pw = 1e-3
    wJiT = pw * Ji.transpose(1, 2) @ W
    wJjT = pw * Jj.transpose(1, 2) @ W
    Hsp = torch.stack([wJiT @ Ji, wJiT @ Jj, wJjT @ Ji, wJjT @ Jj])[:, None].float()
    vsp = (-torch.stack([wJiT @ r, wJjT @ r]).squeeze(-1))[:, None].float()
    out = dict(p)
    out.update(poses=poses, Hsp=Hsp, vsp=vsp, iip=iip, jjp=jjp)
    out = {k: (v.to(device) if isinstance(v, torch.Tensor) else v) for k, v in out.items()}
    out["Hsp"], out["vsp"] = out["Hsp"].contiguous(), out["vsp"].contiguous()
    return out


def make_batch_problems(num_windows=64, seed=0, device="cpu"):
    """The batching workload: ``num_windows`` independent BA windows of uneven sizes --
    keyframes U{8..40}, edges U{20..500} (capped by the K(K-1) ordered pairs), a 43x77
    or 30x40 grid -- each drawn like the frontend window (|i-j| <= 3 pairs first, then
    random pairs), t0 = 1, lm = 1e-4, ep = 0.1.  Returns a list of ``ba`` input dicts."""
    g = torch.Generator().manual_seed(seed + 3000)
    out = []
    for w in range(num_windows):
        K = int(torch.randint(8, 41, (1,), generator=g))
        E = int(torch.randint(20, 501, (1,), generator=g))
        ht, wd, img = (43, 77, (344, 616)) if int(torch.randint(0, 2, (1,), generator=g)) == 0 else (30, 40, (240, 320))
        pairs = [(i, j) for i in range(K) for j in range(K) if i != j]
        near = [p for p in pairs if abs(p[0] - p[1]) <= 3]
        far = [p for p in pairs if abs(p[0] - p[1]) > 3]
        perm = torch.randperm(len(far), generator=g).tolist()
        e = (near + [far[k] for k in perm])[:min(E, len(pairs))]
        intr = intrinsics_for(img)
        xi = 0.05 * torch.randn(K, 6, generator=g, dtype=torch.float64)
        poses_gt = se3_exp(xi)
        disps_gt = 0.1 + 1.9 * torch.rand(K, ht, wd, generator=g, dtype=torch.float64)
        ii = torch.tensor([a for a, _ in e], dtype=torch.int64)
        jj = torch.tensor([b for _, b in e], dtype=torch.int64)
        coords = reproject(poses_gt, disps_gt, intr, ii, jj)
        targets = coords + 0.5 * torch.randn(coords.shape, generator=g, dtype=torch.float64)
        weights = torch.rand(len(e), ht, wd, 2, generator=g, dtype=torch.float64)
        t0 = 1
        poses = poses_gt.clone()
        pert = se3_exp(0.01 * torch.randn(K, 6, generator=g, dtype=torch.float64))
        poses[t0:] = pose_compose(pert[t0:], poses_gt[t0:])
        f32 = dict(dtype=torch.float32, device=device)
        out.append(dict(poses=poses.to(**f32).contiguous(), disps=disps_gt.to(**f32).contiguous(),
                        intrinsics=intr.to(**f32), targets=targets.permute(0, 3, 1, 2).to(**f32).contiguous(),
                        weights=weights.permute(0, 3, 1, 2).to(**f32).contiguous(),
                        eta=torch.full((K, ht, wd), 1e-3, **f32), ii=ii.to(device), jj=jj.to(device), t0=t0, t1=K,
                        iters=4, lm=1e-4, ep=0.1))
    return out


def make_jdsa_problem(name="tiny6", seed=0, device="cpu", hs=2, ws=2, alpha=0.01, keep=None,
                      prior_holes=0.1):
    """Inputs of the mono-prior alignment step ``JDSA`` (``hislam2/geom/ba.py:170``) for the
    BA workload ``name``: its poses, disparities, targets and weights; the edges whose
    source frame passes ``keep`` (default all); ``disps_prior`` [K,H,W] = ground truth
    divided by a smooth per-frame scale field (1 + 0.2 N(0,1) at 3x3 control points,
    bilinear), times 1 + 0.02 N(0,1), with a fraction ``prior_holes`` of pixels set to 0
    (no prior); ``dscales`` [t1,hs,ws] = 1 + 0.05 N(0,1); eta [M,H,W] = 0.2 U[0,1e-2] +
    1e-7 for the M = len(unique(ii)) source frames (the caller's ``.2 * damping + EP``).
    ``alpha`` is ``mono_depth_alpha`` (0.01 in most of HI-SLAM2's configs)."""
    p = make_ba_problem(name, seed=seed, device="cpu")
    g = torch.Generator().manual_seed(seed + 4000)
    K, ht, wd = p["disps"].shape
    t1 = p["t1"]
    ii, jj = p["ii"], p["jj"]
    if keep is not None:
        sel = torch.tensor([bool(keep(int(i))) for i in ii])
        ii, jj = ii[sel], jj[sel]
        p["targets"], p["weights"] = p["targets"][sel].contiguous(), p["weights"][sel].contiguous()
    ctrl = 1.0 + 0.2 * torch.randn(K, 1, 3, 3, generator=g, dtype=torch.float64)
    field = torch.nn.functional.interpolate(ctrl, size=(ht, wd), mode="bilinear", align_corners=True)[:, 0]
    prior = p["disps_gt"].double() / field.clamp(min=0.3)
    prior = prior * (1.0 + 0.02 * torch.randn(K, ht, wd, generator=g, dtype=torch.float64))
    prior = torch.where(torch.rand(K, ht, wd, generator=g) < prior_holes, torch.zeros_like(prior), prior)
    dscales = 1.0 + 0.05 * torch.randn(t1, hs, ws, generator=g, dtype=torch.float64)
    M = int(torch.unique(ii).numel())
    eta = 0.2 * 1e-2 * torch.rand(M, ht, wd, generator=g, dtype=torch.float64) + 1e-7
    f32 = dict(dtype=torch.float32, device=device)
    return dict(targets=p["targets"].to(device), weights=p["weights"].to(device), eta=eta.to(**f32),
                poses=p["poses"][:t1].contiguous().to(device), disps=p["disps"][:t1].contiguous().to(device),
                intrinsics=p["intrinsics"].to(device), disps_prior=prior.to(**f32).contiguous(),
                dscales=dscales.to(**f32).contiguous(), ii=ii.contiguous().to(device),
                jj=jj.contiguous().to(device), alpha=float(alpha))


def make_pgo_factors(poses, iip, jjp, seed=0, noise=0.02):
    """Relative-pose factors between Sim3 poses [K, 8] for the pairs (iip, jjp), in the form
    ``hislam2/depth_video.py:250-256`` passes them to ``global_relative_posesim3_constraints``:
    rel_poses [Np, 7] = the SE3 part (t, q) of Gj Gi^-1, moved by an se3 perturbation
    N(0, noise) so the factors are not at their optimum, and infos [Np, 7, 7] =
    diag(1 / cov, min(1 / cov)) with cov = 10^-U[1, 4] per translational / rotational axis
    (the reference appends the smallest information for the scale)."""
    g = torch.Generator().manual_seed(seed + 5000)
    P = poses.double().cpu()
    pi, pj = P[iip.cpu()], P[jjp.cpu()]
    qi_inv = torch.cat([-pi[:, 3:6], pi[:, 6:7]], -1)
    q = quat_mul(pj[:, 3:7], qi_inv)
    t = pj[:, :3] - (pj[:, 7:8] / pi[:, 7:8]) * quat_rotate(q, pi[:, :3])
    rel = pose_compose(se3_exp(noise * torch.randn(len(iip), 6, generator=g, dtype=torch.float64)),
                       torch.cat([t, q], -1))
    Np = len(iip)
    inv_cov = 10.0 ** (1 + 3 * torch.rand(Np, 6, generator=g, dtype=torch.float64))
    d = torch.cat([inv_cov, inv_cov.min(1, keepdim=True)[0]], 1)
    infos = torch.diag_embed(d)
    return rel.float().to(poses.device).contiguous(), infos.float().to(poses.device).contiguous()
