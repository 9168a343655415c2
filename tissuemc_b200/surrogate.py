"""The learned surrogate: an MLP from layer optical properties to R_d(r), T_t and A, trained on
solves of the batched sweep engine, served behind an ensemble-disagreement gate that routes
untrusted queries back to plain Monte Carlo, and used for inverse fits of mu_a and mu_s'.

There is no counterpart in TissueMC (an addition of this engine). Every arithmetic operation of
the network — forward, backward, loss, Adam — runs in this package's CUDA kernels
(``tmc_b200_nn_*``: tcgen05 tensor-core GEMMs with BF16 operands and FP32 accumulation, fused
bias/GELU epilogues); torch only provides device buffers, random permutations and gathers.

Encoding (13 inputs, 66 outputs):
  inputs   for layer slots 0..2: log10 mu_a, log10 mu_s', g, thickness d (zeros for an absent
           layer: d = 0 marks it), then the shared refractive index n; z-scored, zero-padded to 64.
  outputs  log10 of R_d(r) per unit area [1/cm^2] in the 64 radial bins (floored at 1e-4), then
           T_t and A per photon; z-scored.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import CStatus, CSweepConfig, Layer, _check, lib, sweep_options, sweep_run

N_FEAT, K_IN, HIDDEN, N_HIDDEN = 13, 64, 512, 4
N_RD = 64
N_OUT, N_OUT_PAD = N_RD + 2, 128
RD_FLOOR = 1e-4
LAYER_DIMS = [(K_IN, HIDDEN)] + [(HIDDEN, HIDDEN)] * (N_HIDDEN - 1) + [(HIDDEN, N_OUT_PAD)]  # (in, out)


# ------------------------------------------------------------------------------ encoding
def features(cfgs) -> np.ndarray:
    """(n, 13) raw features of sweep configurations (see the module docstring)."""
    out = np.zeros((len(cfgs), N_FEAT))
    for i, c in enumerate(cfgs):
        for l in range(min(c.num_layers, 3)):
            L = c.layers[l]
            out[i, 4 * l:4 * l + 4] = (math.log10(L.mua), math.log10(L.mus * (1.0 - L.g)), L.g, L.d)
        out[i, 12] = c.layers[0].n
    return out


def annulus_areas(nr: int = N_RD, dr: float = 0.01) -> np.ndarray:
    i = np.arange(nr)
    return math.pi * ((i + 1) ** 2 - i ** 2) * dr * dr


def targets(summary: np.ndarray, dr: float = 0.01) -> np.ndarray:
    """(n, 66) raw targets from sweep summaries (R_d(r) per photon, R_d, T_t, A)."""
    rd_r = summary[:, :N_RD] / annulus_areas(N_RD, dr)
    return np.concatenate([np.log10(np.maximum(rd_r, RD_FLOOR)), summary[:, N_RD + 1:N_RD + 3]], axis=1)


def rd_profile(y_raw: np.ndarray) -> np.ndarray:
    """R_d(r) per unit area from raw (de-normalised) outputs."""
    return 10.0 ** y_raw[..., :N_RD]


def generate(n: int, photons: int, master_seed: int, batch: int = 4096, device: int = 0):
    """n solves of the sweep distribution at a fixed photon count: (configs, X raw, Y raw)."""
    from . import sweep_sample

    cfgs = sweep_sample(master_seed, n)
    for c in cfgs:
        c.photons = photons
    opt = sweep_options(device=device)
    summaries = []
    for s in range(0, n, batch):
        part = (CSweepConfig * min(batch, n - s))(*cfgs[s:s + batch])
        summaries.append(sweep_run(part, opt).summary)
    return cfgs, features(cfgs), targets(np.concatenate(summaries))


# ------------------------------------------------------------------------------ the network
def _call(name, *args):
    st = CStatus()
    _check(getattr(lib(), name)(*args, ctypes.byref(st)), st)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


class Member:
    """One MLP: 4 hidden GELU layers of 512, FP32 master weights with BF16 copies (and their
    transposes for the backward pass), Adam state, and the activations of one batch."""

    def __init__(self, batch: int, seed: int, device: str = "cuda:0"):
        import torch

        self.torch, self.dev, self.B = torch, device, batch
        g = torch.Generator(device="cpu").manual_seed(seed)
        f32, bf = dict(dtype=torch.float32, device=device), dict(dtype=torch.bfloat16, device=device)
        self.W, self.b, self.Wb, self.WT, self.mW, self.vW, self.mb, self.vb, self.gW, self.gb = ([] for _ in range(10))
        for li, (k, n) in enumerate(LAYER_DIMS):
            fan_in = N_FEAT if li == 0 else k
            w = torch.randn(n, k, generator=g) * math.sqrt(2.0 / fan_in)
            if li == 0:
                w[:, N_FEAT:] = 0.0  # padded inputs
            if li == len(LAYER_DIMS) - 1:
                w[N_OUT:, :] = 0.0  # padded outputs
                w *= 0.5
            self.W.append(w.to(**f32).contiguous())
            self.b.append(torch.zeros(n, **f32))
            self.Wb.append(self.W[-1].to(torch.bfloat16).contiguous())
            self.WT.append(self.W[-1].t().contiguous().to(torch.bfloat16))
            for lst, shape in ((self.mW, (n, k)), (self.vW, (n, k)), (self.gW, (n, k))):
                lst.append(torch.zeros(shape, **f32))
            for lst in (self.mb, self.vb, self.gb):
                lst.append(torch.zeros(n, **f32))
        L = len(LAYER_DIMS)
        self.Z = [torch.empty(batch, n, **f32) for (_, n) in LAYER_DIMS]
        self.H = [torch.empty(batch, n, **bf) for (_, n) in LAYER_DIMS[:-1]]
        self.HT = [torch.empty(n, batch, **bf) for (_, n) in LAYER_DIMS[:-1]]
        self.dZ = [torch.empty(batch, n, **bf) for (_, n) in LAYER_DIMS]
        self.dZT = [torch.empty(n, batch, **bf) for (_, n) in LAYER_DIMS]
        self.XT = torch.empty(K_IN, batch, **bf)
        self.loss = torch.zeros(1, **f32)
        self.step_count = 0
        self.L = L

    def forward(self, X, rows: int, stream: int, Z_out=None):
        """X: (rows, 64) bf16 -> the last layer's Z (rows, 128) float32 (into Z_out if given)."""
        h = X
        for li, (k, n) in enumerate(LAYER_DIMS):
            last = li == self.L - 1
            Z = (Z_out if (last and Z_out is not None) else self.Z[li])
            _call("tmc_b200_nn_linear", _p(h), _p(self.Wb[li]), _p(self.b[li]), _p(Z),
                  _p(None if last else self.H[li]), rows, n, k, 0 if last else 1, ctypes.c_void_p(stream))
            if not last:
                h = self.H[li]
        return Z_out if Z_out is not None else self.Z[-1]

    def backward(self, X, Y, stream: int, scale: float):
        """Loss and gradients for one full batch (X: B x 64 bf16, Y: B x 66 float32)."""
        B, s = self.B, ctypes.c_void_p(stream)
        self.loss.zero_()
        _call("tmc_b200_nn_mse", _p(self.Z[-1]), _p(Y), _p(self.dZ[-1]), _p(self.loss), B, N_OUT, N_OUT_PAD,
              ctypes.c_float(scale), s)
        _call("tmc_b200_nn_transpose", _p(X), _p(self.XT), B, K_IN, s)
        for li in range(self.L - 1):
            _call("tmc_b200_nn_transpose", _p(self.H[li]), _p(self.HT[li]), B, LAYER_DIMS[li][1], s)
        for li in range(self.L - 1, -1, -1):
            k, n = LAYER_DIMS[li]
            _call("tmc_b200_nn_transpose", _p(self.dZ[li]), _p(self.dZT[li]), B, n, s)
            prev_T = self.XT if li == 0 else self.HT[li - 1]
            _call("tmc_b200_nn_matmul_f32", _p(self.dZT[li]), _p(prev_T), _p(self.gW[li]), n, k, B, s)
            _call("tmc_b200_nn_colsum", _p(self.dZ[li]), _p(self.gb[li]), B, n, s)
            if li > 0:
                _call("tmc_b200_nn_backward_data", _p(self.dZ[li]), _p(self.WT[li]), _p(self.Z[li - 1]),
                      _p(self.dZ[li - 1]), B, k, n, s)

    def adam(self, stream: int, lr: float, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        self.step_count += 1
        t = self.step_count
        lr_t = lr * math.sqrt(1 - b2 ** t) / (1 - b1 ** t)
        s = ctypes.c_void_p(stream)
        for li, (k, n) in enumerate(LAYER_DIMS):
            _call("tmc_b200_nn_adam", _p(self.W[li]), _p(self.gW[li]), _p(self.mW[li]), _p(self.vW[li]), n, k,
                  ctypes.c_float(lr_t), ctypes.c_float(b1), ctypes.c_float(b2), ctypes.c_float(eps),
                  ctypes.c_float(wd), _p(self.Wb[li]), _p(self.WT[li]), s)
            _call("tmc_b200_nn_adam", _p(self.b[li]), _p(self.gb[li]), _p(self.mb[li]), _p(self.vb[li]), 1, n,
                  ctypes.c_float(lr_t), ctypes.c_float(b1), ctypes.c_float(b2), ctypes.c_float(eps),
                  ctypes.c_float(0.0), _p(None), _p(None), s)


@dataclass
class Norm:
    x_mean: np.ndarray
    x_std: np.ndarray
    y_mean: np.ndarray
    y_std: np.ndarray

    @staticmethod
    def fit(X: np.ndarray, Y: np.ndarray) -> Norm:
        return Norm(X.mean(0), np.maximum(X.std(0), 1e-6), Y.mean(0), np.maximum(Y.std(0), 1e-6))


class Ensemble:
    """Several independently initialised members trained on the same data in different orders."""

    def __init__(self, members: int = 4, batch: int = 4096, seed: int = 0, device: str = "cuda:0"):
        import torch

        self.torch, self.dev, self.B = torch, device, batch
        self.members = [Member(batch, seed * 1000 + i, device) for i in range(members)]
        self.norm: Norm | None = None
        self.history: list[float] = []

    def _x(self, X: np.ndarray):
        t = self.torch
        Xn = np.zeros((len(X), K_IN), dtype=np.float32)
        Xn[:, :N_FEAT] = (X - self.norm.x_mean) / self.norm.x_std
        return t.from_numpy(Xn).to(self.dev).to(t.bfloat16)

    def train(self, X: np.ndarray, Y: np.ndarray, epochs: int, lr: float = 1e-3, seed: int = 0,
              lr_final: float = 1e-5) -> list[float]:
        """Adam with a cosine learning-rate decay; returns the mean training loss per epoch."""
        t = self.torch
        self.norm = Norm.fit(X, Y)
        Xd = self._x(X)
        Yd = t.from_numpy(((Y - self.norm.y_mean) / self.norm.y_std).astype(np.float32)).to(self.dev)
        n = len(X)
        steps = n // self.B
        if steps < 1:
            raise ValueError(f"need at least one full batch of {self.B} samples")
        stream = t.cuda.current_stream().cuda_stream
        gen = t.Generator(device=self.dev).manual_seed(seed)
        scale = 1.0 / (self.B * N_OUT)
        total = epochs * steps
        xb = t.empty(self.B, K_IN, dtype=t.bfloat16, device=self.dev)
        yb = t.empty(self.B, N_OUT, dtype=t.float32, device=self.dev)
        k = 0
        for _ in range(epochs):
            perms = [t.randperm(n, generator=gen, device=self.dev) for _ in self.members]
            acc = t.zeros(1, dtype=t.float32, device=self.dev)
            for s in range(steps):
                lr_k = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * k / total))
                for m, perm in zip(self.members, perms, strict=True):
                    idx = perm[s * self.B:(s + 1) * self.B]
                    t.index_select(Xd, 0, idx, out=xb)
                    t.index_select(Yd, 0, idx, out=yb)
                    m.forward(xb, self.B, stream)
                    m.backward(xb, yb, stream, scale)
                    m.adam(stream, lr_k)
                    acc += m.loss
                k += 1
            self.history.append(float(acc.item()) / (steps * len(self.members)))
        if lib().tmc_b200_nn_status(1):
            raise RuntimeError("a tensor-core wait gave up during training")
        return self.history

    def predict_members(self, X: np.ndarray, chunk: int = 65536) -> np.ndarray:
        """(members, n, 66) raw (de-normalised) outputs."""
        t = self.torch
        stream = t.cuda.current_stream().cuda_stream
        out = np.empty((len(self.members), len(X), N_OUT))
        for s in range(0, len(X), chunk):
            Xc = self._x(X[s:s + chunk])
            rows = len(Xc)
            Z = t.empty(rows, N_OUT_PAD, dtype=t.float32, device=self.dev)
            for i, m in enumerate(self.members):
                _ensure_rows(m, rows)
                m.forward(Xc, rows, stream, Z_out=Z)
                out[i, s:s + rows] = Z[:, :N_OUT].cpu().numpy() * self.norm.y_std + self.norm.y_mean
        return out

    def predict(self, X: np.ndarray) -> np.ndarray:
        return self.predict_members(X).mean(0)


def _ensure_rows(m: Member, rows: int) -> None:
    """Grow a member's activation buffers to `rows` rows for inference."""
    if m.Z[0].shape[0] >= rows:
        return
    t = m.torch
    m.Z = [t.empty(rows, n, dtype=t.float32, device=m.dev) for (_, n) in LAYER_DIMS]
    m.H = [t.empty(rows, n, dtype=t.bfloat16, device=m.dev) for (_, n) in LAYER_DIMS[:-1]]


# ------------------------------------------------------------------------------ the gate
def rd_total(y_raw: np.ndarray, dr: float = 0.01) -> np.ndarray:
    """Diffuse reflectance on the grid (sum of R_d(r) x annulus area) from raw outputs."""
    return (rd_profile(y_raw) * annulus_areas(N_RD, dr)).sum(-1)


def gate(members_out: np.ndarray, threshold: float = 0.01) -> np.ndarray:
    """True where the members disagree: relative spread (max - min) / mean of the predicted
    diffuse reflectance above `threshold` — those queries go back to plain Monte Carlo."""
    rd = rd_total(members_out)
    return (rd.max(0) - rd.min(0)) / np.maximum(rd.mean(0), 1e-12) > threshold


# ------------------------------------------------------------------------------ inverse fit
def lm_fit(ens: Ensemble, base_feats: np.ndarray, obs_log_rd: np.ndarray, mask: np.ndarray, free: list[int],
           iters: int = 30, lam0: float = 1e-2, h: float = 0.03):
    """Levenberg-Marquardt on the features in `free` (columns of the raw feature vector, e.g.
    log10 mu_a and log10 mu_s' of two layers) for a batch of fits at once, through the
    surrogate's Jacobian (central finite differences, all fits and perturbations in one batched
    forward pass per iteration; the step h, in log10 units, is kept well above the BF16 resolution
    of the network's normalised inputs). Residuals: predicted minus observed log10 R_d(r) on the bins in
    `mask`. Returns the fitted features and the final residual norms."""
    theta = base_feats.copy()
    n, p = len(theta), len(free)
    lam = np.full(n, lam0)

    def resid(th):
        y = ens.predict(th)
        return (y[:, :N_RD] - obs_log_rd) * mask

    r = resid(theta)
    cost = (r ** 2).sum(1)
    for _ in range(iters):
        pert = np.repeat(theta[None], 2 * p, 0)
        for j, col in enumerate(free):
            pert[2 * j, :, col] += h
            pert[2 * j + 1, :, col] -= h
        y = ens.predict(pert.reshape(-1, theta.shape[1])).reshape(2 * p, n, -1)[..., :N_RD]
        J = np.stack([(y[2 * j] - y[2 * j + 1]) / (2 * h) * mask for j in range(p)], axis=2)  # n x bins x p
        JtJ = np.einsum("nbi,nbj->nij", J, J)
        Jtr = np.einsum("nbi,nb->ni", J, r)
        A = JtJ + lam[:, None, None] * (np.eye(p)[None] * (np.diagonal(JtJ, axis1=1, axis2=2)[:, :, None] + 1e-9))
        step = -np.linalg.solve(A, Jtr[..., None])[..., 0]
        trial = theta.copy()
        trial[:, free] += np.clip(step, -0.5, 0.5)
        r_new = resid(trial)
        c_new = (r_new ** 2).sum(1)
        better = c_new < cost
        theta[better] = trial[better]
        r[better], cost[better] = r_new[better], c_new[better]
        lam = np.where(better, lam * 0.3, lam * 10.0)
    return theta, np.sqrt(cost)


def config_from_features(f: np.ndarray, photons: int, seed: int) -> CSweepConfig:
    """A sweep configuration from a raw feature vector (inverse of `features`)."""
    c = CSweepConfig()
    c.photons, c.seed, c.n_above, c.n_below = photons, seed, 1.0, 1.0
    nl = 0
    for l in range(3):
        d = f[4 * l + 3]
        if d <= 0:
            break
        g = f[4 * l + 2]
        c.layers[l] = Layer(f[12], 10 ** f[4 * l], 10 ** f[4 * l + 1] / (1 - g), g, d)
        nl += 1
    c.num_layers = nl
    return c
