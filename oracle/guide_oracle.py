"""FP64 restatement of the learned path guide (TEST INFRASTRUCTURE ONLY).

Restates, in double precision with numpy, what the CUDA guide computes
(cuda-raytracer_b200/csrc/guide.cuh, guide.cu), so that its forward outputs
and its gradients can be checked:

* encoding: 12-level hash grid (resolution floor(4 * 1.5**l), direct indexing
  where the lattice fits 2**16 entries, else x plus the xor-of-primes hash of
  y and z),
  2 features per level, trilinear; 16 real SH terms of wo; the normal; zeros
  up to 64 inputs;
* MLP: 5 linear layers 64 -> 64, ReLU after the first four;
* output: 8 vMF lobes (normalised mean, softplus concentration clamped to
  [0.05, 5000], softmax weights);
* loss: sum_r w_r * -log q(w_r) / sum_r w_r, and its exact gradients; with
  learned selection, -log of the one-sample MIS density s q + (1 - s) p_bsdf,
  s the sigmoid of output 40 clamped to [0.02, 0.98].

The reference has no learned component; this module is checked against
finite differences of its own loss (tests/test_oracle_guide.py).
"""
from __future__ import annotations

import numpy as np

LEVELS, FEAT, LOG2T = 12, 2, 16
T = 1 << LOG2T
IN = HID = OUT = 64
LAYERS, LOBES = 5, 8
ENC, SH = LEVELS * FEAT, 16
KMIN, KMAX = 0.05, 5000.0


def grid_res(l):
    r = np.float32(4.0)
    for _ in range(l):
        r = np.float32(r * np.float32(1.5))
    return float(np.floor(r))


def grid_index(l, ix, iy, iz):
    res = int(grid_res(l)) + 1
    if res ** 3 <= T:
        return (ix + res * (iy + res * iz)) & 0xFFFFFFFF
    h = ix + (((iy * 2654435761) & 0xFFFFFFFF) ^ ((iz * 805459861) & 0xFFFFFFFF))
    return h & (T - 1)


def sh16(x, y, z):
    c0, c1 = 0.28209479177387814, 0.4886025119029199
    c2a, c2b, c2c = 1.0925484305920792, 0.31539156525252005, 0.5462742152960396
    c3a, c3b, c3c, c3d, c3e = 0.5900435899266435, 2.890611442640554, 0.4570457994644658, 0.3731763325901154, 1.445305721320277
    xx, yy, zz = x * x, y * y, z * z
    return np.array([c0, -c1 * y, c1 * z, -c1 * x,
                     c2a * x * y, -c2a * y * z, c2b * (3 * zz - 1), -c2a * x * z, c2c * (xx - yy),
                     -c3a * y * (3 * xx - yy), c3b * x * y * z, -c3c * y * (5 * zz - 1), c3d * z * (5 * zz - 3),
                     -c3c * x * (5 * zz - 1), c3e * z * (xx - yy), -c3a * x * (xx - 3 * yy)])


def corners(l, u):
    res = grid_res(l)
    p = np.clip(u, 0.0, 1.0) * res
    f = np.floor(p)
    i = f.astype(np.int64)
    t = p - f
    idx, w = [], []
    for k in range(8):
        d = ((k & 1), (k >> 1) & 1, (k >> 2) & 1)
        idx.append(grid_index(l, int(i[0] + d[0]), int(i[1] + d[1]), int(i[2] + d[2])))
        w.append((t[0] if d[0] else 1 - t[0]) * (t[1] if d[1] else 1 - t[1]) * (t[2] if d[2] else 1 - t[2]))
    return idx, w


def encode(grid, bmin, binv, x, wo, n):
    """grid: (LEVELS, T, FEAT) float64."""
    u = (np.asarray(x, np.float64) - bmin) * binv
    v = np.zeros(IN)
    cs = []
    for l in range(LEVELS):
        idx, w = corners(l, u)
        cs.append((idx, w))
        for k in range(8):
            v[2 * l:2 * l + 2] += w[k] * grid[l, idx[k]]
    v[ENC:ENC + SH] = sh16(*np.asarray(wo, np.float64))
    v[ENC + SH:ENC + SH + 3] = n
    return v, cs


def forward(W, b, h0):
    """W: (LAYERS, 64, 64), b: (LAYERS, 64). Returns output and pre-activations z_1..z_4."""
    zs, h = [], h0
    for l in range(LAYERS):
        z = W[l] @ h + b[l]
        if l == LAYERS - 1:
            return z, zs
        zs.append(z)
        h = np.maximum(z, 0.0)


def softplus(x):
    return x if x > 20 else np.log1p(np.exp(x))


def lobes(o):
    mus, kaps, logits = [], [], []
    for k in range(LOBES):
        m = o[5 * k:5 * k + 3]
        mus.append(m / np.linalg.norm(m))
        kaps.append(min(max(softplus(o[5 * k + 3]), KMIN), KMAX))
        logits.append(o[5 * k + 4])
    logits = np.array(logits)
    w = np.exp(logits - logits.max())
    return np.array(mus), np.array(kaps), w / w.sum()


def vmf(mu, kap, w):
    return kap / (2 * np.pi * (-np.expm1(-2 * kap))) * np.exp(kap * (mu @ w - 1))


def log_vmf(mu, kap, w):
    return np.log(kap / (2 * np.pi)) - np.log1p(-np.exp(-2 * kap)) + kap * (mu @ w - 1)


def log_terms(o, w):
    """log(pi_k v_k(w)) per lobe and their log-sum-exp, log q(w): in log space,
    so that directions far from every sharp lobe keep their responsibilities."""
    mus, kaps, pis = lobes(o)
    with np.errstate(divide="ignore"):
        lv = np.array([np.log(pis[k]) + log_vmf(mus[k], kaps[k], w) for k in range(LOBES)])
    mx = lv.max()
    return lv, mx + np.log(np.exp(lv - mx).sum())


def mixture_pdf(o, w):
    return np.exp(log_terms(o, w)[1])


def nll_grad(o, w, scale):
    """d(-scale * log q(w)) / d o  (first 40 outputs; the rest are zero)."""
    mus, kaps, pis = lobes(o)
    lv, logq = log_terms(o, w)
    g = np.zeros(OUT)
    for k in range(LOBES):
        gam = np.exp(lv[k] - logq)
        g[5 * k + 4] = scale * (pis[k] - gam)
        raw = o[5 * k + 3]
        sp = softplus(raw)
        clamped = sp < KMIN or sp > KMAX
        kap = kaps[k]
        dlogv = 1 / kap - 2 * np.exp(-2 * kap) / -np.expm1(-2 * kap) + mus[k] @ w - 1  # 2 / (e^{2 kappa} - 1)
        sig = 1 / (1 + np.exp(-raw))
        g[5 * k + 3] = 0.0 if clamped else -scale * gam * dlogv * sig
        m = o[5 * k:5 * k + 3]
        ln = np.linalg.norm(m)
        g[5 * k:5 * k + 3] = -scale * gam * kap * (w - mus[k] * (mus[k] @ w)) / ln
    return g


# Learned selection: output SEL_OUT is the logit of the probability of sampling
# the guide (rather than the BSDF) at a vertex, clamped to [SEL_MIN, SEL_MAX].
# The loss then fits the one-sample MIS density m = s q + (1 - s) p_bsdf that
# the renderer samples with (the objective of Mueller et al. 2019 applied to
# the whole mixture), so that q and s are trained together.
SEL_OUT, SEL_MIN, SEL_MAX = 40, 0.02, 0.98


def selection(o):
    raw = 1 / (1 + np.exp(-o[SEL_OUT]))
    return min(max(raw, SEL_MIN), SEL_MAX), SEL_MIN < raw < SEL_MAX


def log_density(o, w, pb, learn_select):
    """The log of the density the loss fits: q(w), or s q(w) + (1 - s) p_bsdf."""
    logq = log_terms(o, w)[1]
    if not learn_select:
        return logq
    s, _ = selection(o)
    return np.logaddexp(np.log(s) + logq, np.log(1 - s) + np.log(pb) if pb > 0 else -np.inf)


def nll_grad_select(o, w, pb, scale):
    """d(-scale * log(s q(w) + (1 - s) pb)) / d o."""
    logq = log_terms(o, w)[1]
    s, free = selection(o)
    r = np.exp(np.log(s) + logq - log_density(o, w, pb, True))  # the guide's share s q / m
    g = nll_grad(o, w, scale) * r
    g[SEL_OUT] = -scale * ((1 - s) * r - s * (1 - r)) if free else 0.0
    return g


def _pb(r):
    return r[13] if len(r) > 13 else 0.0


def loss(grid, W, b, bmin, binv, records, learn_select=False):
    """Weighted NLL of records (n x 13: x, wo, n, w, weight; a 14th value, the
    BSDF density of w, with learned selection), normalised."""
    tot = sum(r[12] for r in records if r[12] > 0)
    s = 0.0
    for r in records:
        if r[12] <= 0:
            continue
        h0, _ = encode(grid, bmin, binv, r[0:3], r[3:6], r[6:9])
        o, _ = forward(W, b, h0)
        s += r[12] * -log_density(o, r[9:12], _pb(r), learn_select)
    return s / tot


def out_grad(o, r, scale, learn_select):
    w = np.asarray(r[9:12], np.float64)
    return nll_grad_select(o, w, _pb(r), scale) if learn_select else nll_grad(o, w, scale)


def gradients(grid, W, b, bmin, binv, records, learn_select=False):
    """Exact gradients of `loss` with respect to W, b and the grid."""
    gW, gb, ggrid = np.zeros_like(W), np.zeros_like(b), np.zeros_like(grid)
    tot = sum(r[12] for r in records if r[12] > 0)
    for r in records:
        if r[12] <= 0:
            continue
        h0, cs = encode(grid, bmin, binv, r[0:3], r[3:6], r[6:9])
        o, zs = forward(W, b, h0)
        dz = out_grad(o, r, r[12] / tot, learn_select)
        for l in range(LAYERS - 1, -1, -1):
            h = h0 if l == 0 else np.maximum(zs[l - 1], 0.0)
            gW[l] += np.outer(dz, h)
            gb[l] += dz
            dh = W[l].T @ dz
            if l > 0:
                dz = dh * (zs[l - 1] > 0)
            else:
                for lv, (idx, w) in enumerate(cs):
                    for k in range(8):
                        ggrid[lv, idx[k]] += w[k] * dh[2 * lv:2 * lv + 2]
    return gW, gb, ggrid


# ---------------------------------------------------------------------------
# BF16 emulation of the tensor-core passes (cuda-raytracer_b200/csrc/guide_tc.cuh
# and k_guide_train_tc): the same arithmetic in FP64 with the operands rounded
# to BF16 (round to nearest even) where the kernels round them: the encoding and
# the hidden activations, the weights, and the output gradient of every layer as
# it enters the two backward products.  Biases, accumulations, bias gradients and
# the ReLU masks stay unrounded.

def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(a, np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(W, b, h0):
    """Forward pass as the tensor cores compute it; returns the output and the
    BF16 layer inputs h_0..h_4."""
    Wb = bf16(W)
    hs, h = [], bf16(h0)
    for l in range(LAYERS):
        hs.append(h)
        z = Wb[l] @ h + b[l]
        if l == LAYERS - 1:
            return z, hs
        h = bf16(np.maximum(z, 0.0))


def gradients_bf16(grid, W, b, bmin, binv, records, learn_select=False):
    """Gradients of `loss` as the tensor-core training pass forms them."""
    gW, gb, ggrid = np.zeros_like(W), np.zeros_like(b), np.zeros_like(grid)
    Wb = bf16(W)
    tot = sum(r[12] for r in records if r[12] > 0)
    for r in records:
        if r[12] <= 0:
            continue
        h0, cs = encode(grid, bmin, binv, r[0:3], r[3:6], r[6:9])
        o, hs = forward_bf16(W, b, h0)
        dz = out_grad(o, r, r[12] / tot, learn_select)
        for l in range(LAYERS - 1, -1, -1):
            dzb = bf16(dz)
            gW[l] += np.outer(dzb, hs[l])
            gb[l] += dz
            dh = Wb[l].T @ dzb
            if l > 0:
                dz = dh * (hs[l] > 0)
            else:
                for lv, (idx, w) in enumerate(cs):
                    for k in range(8):
                        ggrid[lv, idx[k]] += w[k] * dh[2 * lv:2 * lv + 2]
    return gW, gb, ggrid
