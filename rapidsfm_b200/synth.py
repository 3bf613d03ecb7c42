"""Seeded synthetic SIFT-like descriptors (128 x uint8), as specified for the matcher workloads.

Each descriptor: 128 half-normal(sigma=1) floats, L2-normalised, clipped at 0.2, renormalised,
scaled by 512, rounded and clamped to [0, 255]. A train set holds noisy copies (add N(0, sigma),
requantise to [0, 255]) of a fraction of the query descriptors in shuffled order; the rest are
independent descriptors. Randomness: numpy.random.Generator(PCG64(seed)).
"""
import numpy as np


def _sift_like(rng, n):
    x = np.abs(rng.standard_normal((n, 128), dtype=np.float32))
    x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
    np.minimum(x, 0.2, out=x)
    x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
    x *= 512.0
    return np.clip(np.rint(x), 0, 255).astype(np.uint8)


def make_pair(n_query, n_train, overlap, sigma, seed):
    """Returns (query uint8[nq,128], train uint8[nt,128], truth int64[nt]).

    truth[j] is the query index train descriptor j was copied from, or -1 for independent ones.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    q = _sift_like(rng, n_query)
    n_copy = int(round(overlap * min(n_query, n_train)))
    src = rng.choice(n_query, size=n_copy, replace=False) if n_copy > 0 else np.zeros(0, dtype=np.int64)
    copies = q[src].astype(np.float32) + rng.normal(0.0, sigma, size=(n_copy, 128)).astype(np.float32)
    copies = np.clip(np.rint(copies), 0, 255).astype(np.uint8)
    indep = _sift_like(rng, n_train - n_copy)
    t = np.concatenate([copies, indep], axis=0)
    truth = np.concatenate([src.astype(np.int64), np.full(n_train - n_copy, -1, dtype=np.int64)])
    perm = rng.permutation(n_train)
    return q, t[perm], truth[perm]


def uniform_bytes(n, seed):
    """Uniform random bytes (the reference's kernel tests use uniform random 32-bit words)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.integers(0, 256, size=(n, 128), dtype=np.uint8)


def _sift_like_torch(n, gen, device):
    import torch
    x = torch.randn((n, 128), generator=gen, device=device, dtype=torch.float32).abs_()
    x /= x.norm(dim=1, keepdim=True).clamp_min_(1e-12)
    x.clamp_max_(0.2)
    x /= x.norm(dim=1, keepdim=True).clamp_min_(1e-12)
    return (x * 512.0).round_().clamp_(0, 255).to(torch.uint8)


def make_pair_torch(n_query, n_train, overlap, sigma, gen, device="cuda"):
    """make_pair's distribution drawn on the device from a torch.Generator (large batched
    workloads, where host generation would dominate). Returns CUDA tensors (query, train, truth)."""
    import torch
    q = _sift_like_torch(n_query, gen, device)
    n_copy = int(round(overlap * min(n_query, n_train)))
    src = torch.randperm(n_query, generator=gen, device=device)[:n_copy]
    noise = torch.randn((n_copy, 128), generator=gen, device=device) * sigma
    copies = (q[src].float() + noise).round_().clamp_(0, 255).to(torch.uint8)
    t = torch.cat([copies, _sift_like_torch(n_train - n_copy, gen, device)])
    truth = torch.cat([src, torch.full((n_train - n_copy,), -1, dtype=torch.int64, device=device)])
    perm = torch.randperm(n_train, generator=gen, device=device)
    return q, t[perm].contiguous(), truth[perm]


def make_ransac_matches(n, width=1600, height=1200, inlier_frac=0.7, noise=1.0, seed=0, cluster=None):
    """Synthetic point matches for the RANSAC match filter: float32 [n, 4] (lx, ly, rx, ry) and the
    true inlier mask. Inliers follow a smooth warp (similarity plus a gentle perspective bend) with
    Gaussian noise; outliers have uniform random right points. cluster=(x, y, r): left points
    drawn in that disc instead of the whole image (dense cells)."""
    rng = np.random.default_rng(seed)
    if cluster is None:
        left = rng.uniform((0, 0), (width, height), (n, 2))
    else:
        cx, cy, r = cluster
        ang = rng.uniform(0, 2 * np.pi, n)
        rad = r * np.sqrt(rng.uniform(0, 1, n))
        left = np.stack([cx + rad * np.cos(ang), cy + rad * np.sin(ang)], 1)
    th = np.deg2rad(rng.uniform(-15, 15))
    s = rng.uniform(0.8, 1.25)
    R = s * np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    t = rng.uniform(-100, 100, 2)
    c = left - (width / 2, height / 2)
    bend = 1.0 + 2e-5 * (c[:, :1] * rng.uniform(-1, 1) + c[:, 1:] * rng.uniform(-1, 1))
    right = (c @ R.T) / bend + (width / 2, height / 2) + t + rng.normal(0, noise, (n, 2))
    inl = rng.uniform(0, 1, n) < inlier_frac
    right[~inl] = rng.uniform((0, 0), (width, height), ((~inl).sum(), 2))
    return np.concatenate([left, right], 1).astype(np.float32), inl
