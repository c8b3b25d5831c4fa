"""CPU oracle of the learned seed pruner (test infrastructure only).

Restates, in numpy, what the CUDA kernels of allen_b200/csrc/velo_mlp.cuh and velo_mlp.cu
compute, with the same rounding points, so the GPU features, logits and gradients can be
checked against it:

* doublet_features(): the 12 fp32 doublet features, operation for operation (IEEE division
  and square root are correctly rounded in both, and the kernels are built without FMA
  contraction), so they agree bit for bit;
* forward() / gradients(): the 12-32-32-1 network with bf16 (round to nearest even) inputs,
  weights and layer inputs and fp32 biases; sums in float64 here, fp32 in the tensor-core
  kernels, so results agree to rounding of the sums.

The pruner has no counterpart in the reference (its seeding is SearchByTriplet.cu:298-446);
the training labels come from the plain search, which is itself pinned bit for bit against
the reference CPU build.
"""
import numpy as np

N_FEATURES = 12
HIDDEN = 32
N_PARAMS = HIDDEN * N_FEATURES + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN + 1
RECORD_DTYPE = np.dtype([("f", np.float32, (N_FEATURES,)), ("label", np.float32), ("event", np.uint32),
                         ("h0", np.uint32), ("h1", np.uint32)])


def bf16(a):
    """float32 -> nearest bf16 (ties to even), returned as float32 values."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def doublet_features(x0, y0, z0, phi0, x1, y1, z1, phi1, rank, found):
    """Arrays of float32 positions and int16 phi of h0 and h1 -> [n, 12] float32."""
    f32 = np.float32
    x0, y0, z0, x1, y1, z1 = (np.asarray(v, f32) for v in (x0, y0, z0, x1, y1, z1))
    phi0 = np.asarray(phi0, np.int16)
    phi1 = np.asarray(phi1, np.int16)
    with np.errstate(divide="ignore", invalid="ignore"):
        dz = z1 - z0
        inv = f32(1.0) / dz
        tx = (x1 - x0) * inv
        ty = (y1 - y0) * inv
        t2 = tx * tx + ty * ty
        t = np.sqrt(t2)
        doca = (x1 * ty - y1 * tx) / np.maximum(t, f32(1e-6))
        zpoca = z1 - (x1 * tx + y1 * ty) / np.maximum(t2, f32(1e-12))
        r0 = np.sqrt(x0 * x0 + y0 * y0)
        r1 = np.sqrt(x1 * x1 + y1 * y1)
        dphi = (phi1.astype(np.int32) - phi0.astype(np.int32)).astype(np.int16).astype(f32)
        out = np.stack([tx, ty, t, doca, zpoca, dphi * f32(3.0517578125e-05), r1, (r1 - r0) * inv, np.abs(dz),
                        np.asarray(rank, f32), np.asarray(found, f32), phi1.astype(f32) * f32(3.0517578125e-05)],
                       axis=-1)
    return out.astype(f32)


def split(params):
    p = np.asarray(params, np.float32)
    o = 0
    w1 = p[o:o + HIDDEN * N_FEATURES].reshape(HIDDEN, N_FEATURES); o += HIDDEN * N_FEATURES
    b1 = p[o:o + HIDDEN]; o += HIDDEN
    w2 = p[o:o + HIDDEN * HIDDEN].reshape(HIDDEN, HIDDEN); o += HIDDEN * HIDDEN
    b2 = p[o:o + HIDDEN]; o += HIDDEN
    w3 = p[o:o + HIDDEN]; o += HIDDEN
    return w1, b1, w2, b2, w3, p[o]


def standardise(f, mean, inv_std):
    f32 = np.float32
    v = (np.asarray(f, f32) - np.asarray(mean, f32)) * np.asarray(inv_std, f32)
    return np.minimum(np.maximum(v, f32(-8.0)), f32(8.0))


def _round(a, rounding):
    return bf16(np.asarray(a, np.float32)).astype(np.float64) if rounding else np.asarray(a, np.float64)


def forward(params, mean, inv_std, f, rounding=True):
    """Logits and intermediates of the network on raw features f [n, 12].  rounding=False
    drops the bf16 rounding (exact float64 math, for finite-difference checks)."""
    w1, b1, w2, b2, w3, b3 = split(params) if rounding else [np.asarray(v, np.float64) for v in _split64(params)]
    x = _round(standardise(f, mean, inv_std), rounding)
    W1, W2, W3 = (_round(w, rounding) for w in (w1, w2, w3))
    h1 = x @ W1.T + b1
    a2 = _round(np.maximum(h1, 0), rounding)
    h2 = a2 @ W2.T + b2
    a3 = _round(np.maximum(h2, 0), rounding)
    z = a3 @ W3 + float(b3)
    return z, (x, h1, a2, h2, a3, W2, W3)


def _split64(params):
    p = np.asarray(params, np.float64)
    o, out = 0, []
    for size, shape in ((HIDDEN * N_FEATURES, (HIDDEN, N_FEATURES)), (HIDDEN, None), (HIDDEN * HIDDEN, (HIDDEN, HIDDEN)),
                        (HIDDEN, None), (HIDDEN, None), (1, None)):
        v = p[o:o + size]
        out.append(v.reshape(shape) if shape else (v if size > 1 else v[0]))
        o += size
    return out


def gradients(params, mean, inv_std, f, label, pos_weight=1.0, rounding=True):
    """Mean weighted binary cross-entropy and its gradient (flat, parameter order), with the
    kernels' bf16 rounding of the back-propagated layer gradients (rounding=True)."""
    z, (x, h1, a2, h2, a3, W2, W3) = forward(params, mean, inv_std, f, rounding)
    y = np.asarray(label, np.float64)
    n = len(y)
    w = np.where(y > 0.5, pos_weight, 1.0)
    loss = np.sum(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))) / n
    dz = w * (1.0 / (1.0 + np.exp(-z)) - y) / n
    g_w3 = dz @ a3
    g_b3 = dz.sum()
    d2 = np.where(h2 > 0, dz[:, None] * W3[None, :], 0.0)
    g_b2 = d2.sum(0)
    e2 = _round(d2, rounding)
    g_w2 = e2.T @ a2
    d1 = np.where(h1 > 0, e2 @ W2, 0.0)
    g_b1 = d1.sum(0)
    e1 = _round(d1, rounding)
    g_w1 = e1.T @ x
    grad = np.concatenate([g_w1.ravel(), g_b1, g_w2.ravel(), g_b2, g_w3, [g_b3]])
    return loss, grad
