"""Learned hash projection (no reference counterpart): a 128 -> 256 -> 128 MLP whose output signs
replace cascade hashing's random projections (casHash/computeHash.cu) as bucket keys and the
128-bit ranking code.

    x = desc / 64;  h = bf16(relu(W1 x + b1));  o = W2 h + b2;  bit c = [o_c > 0]
    bucket key of table s = bits 8s..8s+7 (bytes 0..7 of the code); code = all 128 bits

Parameters live in one float32 block w1 [256*128] | b1 [256] | w2 [128*256] | b2 [128]. Training
(triplet loss on tanh(o), Adam) and inference run on the GPU through the C ABI
(rsfm_mlp_trainer_*, rsfm_mlp_hash); triplets come from brute-force matches (bf_match_ext).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .matcher import BFTask, bf_match_ext, _check_desc, _stream_ptr

SIZES = (256 * 128, 256, 128 * 256, 128)
NPARAMS = sum(SIZES)


def split(params):
    out, o = [], 0
    for n in SIZES:
        out.append(params[o:o + n])
        o += n
    return out


def init_params(seed=0):
    """He-style initialisation (biases zero) as a float32 parameter block."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0.0, 0.1, size=256 * 128)  # x = desc/64 has norm ~8: pre-activations of std ~0.8
    w2 = rng.normal(0.0, np.sqrt(2.0 / 256), size=128 * 256)
    return np.concatenate([w1, np.zeros(256), w2, np.zeros(128)]).astype(np.float32)


class LearnedHash:
    """Inference handle over device weights (bf16 w1/w2, f32 biases)."""

    def __init__(self, params=None, device="cuda", model=None, keep=None):
        self._keep = keep  # owner of the device memory when `model` is a trainer's view
        if model is not None:
            self.model = model
            return
        p = np.asarray(params, dtype=np.float32)
        w1, b1, w2, b2 = split(p)
        dev = torch.device(device)
        self._w1 = torch.from_numpy(w1.copy()).to(dev).to(torch.bfloat16).contiguous()
        self._w2 = torch.from_numpy(w2.copy()).to(dev).to(torch.bfloat16).contiguous()
        self._b1 = torch.from_numpy(b1.copy()).to(dev)
        self._b2 = torch.from_numpy(b2.copy()).to(dev)
        self.model = _lib.MLP(self._w1.data_ptr(), self._b1.data_ptr(), self._w2.data_ptr(), self._b2.data_ptr())

    def hash(self, desc, keys=None, codes=None, outputs=False, stream=None):
        """desc uint8 [n,128] (CUDA) -> (keys uint8 [n,8], codes int32 [n,4], outputs f32 [n,128] or None)."""
        _check_desc(desc)
        n = desc.shape[0]
        dev = desc.device
        keys = torch.empty((n, 8), dtype=torch.uint8, device=dev) if keys is None else keys
        codes = torch.empty((n, 4), dtype=torch.int32, device=dev) if codes is None else codes
        out = torch.empty((n, 128), dtype=torch.float32, device=dev) if outputs else None
        lib = _lib.load()
        _lib.check(lib.rsfm_mlp_hash(ctypes.byref(self.model), ctypes.c_void_p(desc.data_ptr()), n,
                                     ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(codes.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr() if out is not None else 0), _stream_ptr(stream)),
                   "rsfm_mlp_hash")
        return keys, codes, out


class Trainer:
    """GPU triplet trainer (rsfm_mlp_trainer_*): fp32 masters + Adam, bf16 copies for inference."""

    def __init__(self, params, batch, lr=1e-3, margin=0.5, loss="triplet", lam=16.0):
        lib = _lib.load()
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != NPARAMS:
            raise ValueError("parameter block must hold %d floats" % NPARAMS)
        self.batch = batch
        self._h = ctypes.c_void_p(0)
        _lib.check(lib.rsfm_mlp_trainer_create(p.ctypes.data, batch, lr, margin, ctypes.byref(self._h)),
                   "rsfm_mlp_trainer_create")
        if loss not in ("triplet", "bucket"):
            raise ValueError("loss must be 'triplet' or 'bucket'")
        _lib.check(lib.rsfm_mlp_trainer_set_loss(self._h, 1 if loss == "bucket" else 0, lam),
                   "rsfm_mlp_trainer_set_loss")
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")

    @staticmethod
    def _args(a, ia, p, ip, n, in_):
        return [ctypes.c_void_p(x.data_ptr()) for x in (a, ia, p, ip, n, in_)]

    def step(self, a, ia, p, ip, n, in_, stream=None):
        """One Adam step on the triplets (a[ia[b]], p[ip[b]], n[in_[b]]); loss left in self.loss."""
        _lib.check(_lib.load().rsfm_mlp_trainer_step(self._h, *self._args(a, ia, p, ip, n, in_),
                                                     ctypes.c_void_p(self.loss.data_ptr()), _stream_ptr(stream)),
                   "rsfm_mlp_trainer_step")

    def gradients(self, a, ia, p, ip, n, in_, stream=None):
        g = np.empty(NPARAMS, dtype=np.float32)
        loss = ctypes.c_float(0)
        _lib.check(_lib.load().rsfm_mlp_trainer_gradients(self._h, *self._args(a, ia, p, ip, n, in_),
                                                          g.ctypes.data, ctypes.byref(loss), _stream_ptr(stream)),
                   "rsfm_mlp_trainer_gradients")
        return float(loss.value), g

    def params(self):
        out = np.empty(NPARAMS, dtype=np.float32)
        _lib.check(_lib.load().rsfm_mlp_trainer_params(self._h, out.ctypes.data), "rsfm_mlp_trainer_params")
        return out

    def hasher(self):
        m = _lib.MLP()
        _lib.check(_lib.load().rsfm_mlp_trainer_model(self._h, ctypes.byref(m)), "rsfm_mlp_trainer_model")
        return LearnedHash(model=m, keep=self)

    def close(self):
        if self._h:
            _lib.load().rsfm_mlp_trainer_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class StepGraph:
    """`body` (one trainer step, including the caller's sampling of its index tensors on the
    device) captured once in a CUDA graph and replayed: one launch per step instead of one per
    kernel. `generators`: torch generators that `body` draws from (their state advances on every
    replay). `body` runs `warmup` times eagerly first (lazy initialisation happens outside the
    capture); tensors it allocates during the capture keep their addresses on every replay."""

    def __init__(self, body, generators=(), warmup=3):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                body()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        for g in generators:
            self.graph.register_generator_state(g)
        with torch.cuda.graph(self.graph):
            body()

    def replay(self):
        self.graph.replay()


def center_output_bias(params, hasher_factory, sample_desc):
    """Sets b2 so every output bit splits `sample_desc` in half (median of o before the bias)."""
    p = np.array(params, dtype=np.float32, copy=True)
    w1, b1, w2, b2 = split(p)
    b2[:] = 0
    h = hasher_factory(p)
    _, _, out = h.hash(sample_desc, outputs=True)
    b2[:] = -np.median(out.cpu().numpy(), axis=0)
    return p


def mine_correspondences(pairs, ratio_num=64, ratio_den=100):
    """Brute-force matches that pass the ratio test and the cross-check, per (query, train) pair of
    CUDA descriptor tensors: list of (query index tensor, train index tensor) on the device."""
    tasks = [BFTask(q, t) for q, t in pairs]
    bf_match_ext(tasks, ratio_num, ratio_den)
    out = []
    for t in tasks:
        ok = (t.flagsA & 3) == 3
        qi = torch.nonzero(ok).flatten().to(torch.int32)
        ti = (t.bestA[ok.bool()] & 0xFFFFFFFF).to(torch.int32)
        out.append((qi, ti))
    return out


def default_params_path():
    """Trained parameter block shipped with the package (written by `python -m
    rapidsfm_b200.learned_hash --out <path>`)."""
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "learned_hash_params.npy")


def train_from_brute_force(n_pairs=200, n=8192, steps=20000, batch=4096, lr=1e-3, margin=48.0, seed=0,
                           device="cuda", log=None, loss="triplet", lam=16.0, timings=None):
    """Trains the learned hash on correspondences the brute-force matcher produces (ratio test and
    cross-check passed) on `n_pairs` seeded synthetic pairs (40% overlap, noise 8); negatives are
    random train descriptors of the same pair. Returns the f32 parameter block. `timings` (a dict)
    receives the wall time of the mining and of the training loop."""
    import time
    from . import synth
    t0 = time.perf_counter()
    g = torch.Generator(device=device)
    g.manual_seed(seed + 12345)
    qs, ts, A, P = [], [], [], []
    for k in range(n_pairs):
        q, t, _ = synth.make_pair_torch(n, n, 0.4, 8.0, g, device)
        (qi, ti), = mine_correspondences([(q, t)])
        qs.append(q)
        ts.append(t)
        A.append(qi + k * n)
        P.append(ti + k * n)
    Q, T = torch.cat(qs), torch.cat(ts)
    A, P = torch.cat(A), torch.cat(P)
    params = center_output_bias(init_params(seed), lambda p: LearnedHash(p, device=device), Q[:20000])
    tr = Trainer(params, batch, lr=lr, margin=margin, loss=loss, lam=lam)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    def one():
        sel = torch.randint(0, len(A), (batch,), device=device, generator=g)
        ip = P[sel].int()
        inn = ((ip // n) * n + torch.randint(0, n, (batch,), device=device, generator=g)).int()
        tr.step(Q, A[sel].int(), T, ip, T, inn)

    # the first steps run eagerly (warm-up), the rest from a CUDA graph of one step
    warm = 3
    if steps > warm:
        graph = StepGraph(one, generators=(g,), warmup=warm)
        for s in range(warm, steps):
            graph.replay()
            if log and (s % 1000 == 0 or s == steps - 1):
                log(f"step {s} loss {tr.loss.item():.4f}")
    else:
        for _ in range(steps):
            one()
    out = tr.params()
    tr.close()
    if timings is not None:
        timings["mining_s"] = t1 - t0
        timings["training_loop_s"] = time.perf_counter() - t1
        timings["steps"] = steps
        timings["batch"] = batch
        timings["correspondences"] = int(len(A))
    return out


if __name__ == "__main__":
    import argparse
    import os
    ap = argparse.ArgumentParser(description="train the learned hash on brute-force correspondences")
    ap.add_argument("--out", default=default_params_path())
    ap.add_argument("--pairs", type=int, default=200)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--margin", type=float, default=48.0)
    ap.add_argument("--loss", default="triplet", choices=["triplet", "bucket"])
    ap.add_argument("--lam", type=float, default=16.0)
    a = ap.parse_args()
    p = train_from_brute_force(a.pairs, steps=a.steps, batch=a.batch, margin=a.margin, log=print, loss=a.loss,
                               lam=a.lam)
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.save(a.out, p)
    print("saved", a.out)
