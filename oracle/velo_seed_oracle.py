"""CPU oracle of the learned seed pruner (test infrastructure only).

Restates, in numpy, what the CUDA kernels of allen_b200/csrc/velo_gate.cu, velo_mlp.cuh and
velo_mlp.cu compute, with the same rounding points, so the GPU features, logits and gradients can be
checked against it:

* seed_features(): the 12 fp32 features of a seed candidate, operation for operation (IEEE
  division and square root are correctly rounded in both, and the kernels are built without
  FMA contraction), so they agree bit for bit;
* forward() / gradients(): the 12-32-32-1 network with bf16 (round to nearest even) inputs,
  weights and layer inputs and fp32 biases; sums in float64 here, fp32 in the tensor-core
  kernels, so results agree to rounding of the sums.

The gate has no counterpart in the reference (its seeding is SearchByTriplet.cu:298-446);
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


F32 = np.float32
PI_F = F32(3.141592654)
CONVERT_I16 = F32(32768.0) / PI_F
C1 = F32(0.25) * PI_F
C2 = F32(0.75) * PI_F


def float_to_i16(v):
    """float -> int16 through a 32-bit truncation toward zero (VeloTools.cuh:55-60)."""
    return np.int16(np.int32(np.trunc(v)).astype(np.int16))


def fast_atan2f(y, x):
    """VeloTools.cuh:18-38, fp32 operation for operation."""
    y, x = F32(y), F32(x)
    abs_y = F32(abs(y))
    nom = (x - abs_y) if x > 0 else (x + abs_y)
    den = (x + abs_y) if x > 0 else (abs_y - x)
    r = F32(nom / den)
    angle = (C1 if x > 0 else C2) - C1 * r
    return F32(np.copysign(angle, y))


def hit_phi_16(x, y):
    return float_to_i16(fast_atan2f(y, x) * CONVERT_I16)


def phi_tolerance_i16(phi_tolerance=0.045):
    return int(np.int32(np.trunc(F32(phi_tolerance) * CONVERT_I16)).astype(np.int16))


def leftmost(phis, value):
    """binary_search_leftmost (BinarySearch.cuh:15-30): first index with phi >= value."""
    return int(np.searchsorted(phis.astype(np.int32), int(value), side="left"))


def module_zs(geometry: bytes):
    """The 52 module z of velo_geometry.bin (count, then floats)."""
    n = int(np.frombuffer(geometry[:8], np.uint64)[0])
    return np.frombuffer(geometry[8:8 + 4 * n], np.float32)


def seed_features(xyz, phi, start, num, zs, m, h1, tol):
    """The 12 features of seed candidate h1 (event-relative index into xyz [n, 3] float32 and phi
    int16 of the event's sorted hits) on module pair m = 1..24; start / num: the event's module
    pair offsets (event-relative) and cluster counts; zs: module z; tol: the phi tolerance as
    int16.  The kernel's seed_features (allen_b200/csrc/velo_gate.cu), fp32 operation for
    operation."""
    def hit(i):
        return F32(xyz[i, 0]), F32(xyz[i, 1]), F32(xyz[i, 2])

    x1, y1, z1 = hit(h1)
    phi1 = int(phi[h1])
    ps, pn = int(start[m + 1]), int(num[m + 1])
    ns, nn = int(start[m - 1]), int(num[m - 1])
    pphi, nphi = phi[ps:ps + pn], phi[ns:ns + nn]
    best_d = second_d = F32(1000.0)
    best_z = best_t = F32(0.0)
    min_dphi = F32(1.0)
    best = second = None
    pos = leftmost(pphi, phi1)
    for i in range(min(pn, 4)):
        pos += i if (i & 1) else -i
        ib = pos + pn if pos < 0 else (pos - pn if pos >= pn else pos)
        h0 = ps + ib
        x0, y0, z0 = hit(h0)
        inv = F32(1.0) / (z1 - z0)
        tx = (x1 - x0) * inv
        ty = (y1 - y0) * inv
        t2 = tx * tx + ty * ty
        t = F32(np.sqrt(t2))
        d = F32(abs(x1 * ty - y1 * tx)) / max(t, F32(1e-6))
        dphi = F32(abs(int(np.int16(np.int32(phi1) - np.int32(phi[h0]))))) * F32(3.0517578125e-05)
        min_dphi = min(min_dphi, dphi)
        if d < best_d:
            second_d, second = best_d, best
            best_d, best = d, (h0, tx, ty)
            best_z = z1 - (x1 * tx + y1 * ty) / max(t2, F32(1e-12))
            best_t = t
        elif d < second_d:
            second_d, second = d, (h0, tx, ty)
    dz_next = F32(zs[2 * (m - 1)]) - F32(zs[2 * (m + 1)])
    scatter = [F32(1000.0), F32(1000.0)]
    for c, cand in enumerate((best, second)):
        if cand is None or nn == 0:
            continue
        h0, tx, ty = cand
        x0, y0, z0 = hit(h0)
        xp = x0 + tx * dz_next
        yp = y0 + ty * dz_next
        phi_p = int(hit_phi_16(xp, yp))
        lo = int(np.int16(np.int32(phi_p) - np.int32(tol)))
        st = int(np.int16(leftmost(nphi, lo)))
        idx = (st & 0xFFFFFFFF) % nn
        for _ in range(min(nn, 3)):
            h2 = ns + idx
            if abs(int(np.int16(np.int32(phi[h2]) - np.int32(phi_p)))) > tol:
                break
            x2, y2, z2 = hit(h2)
            dz = z2 - z0
            dx = (x0 + tx * dz) - x2
            dy = (y0 + ty * dz) - y2
            scatter[c] = min(scatter[c], dx * dx + dy * dy)
            idx = 0 if idx + 1 == nn else idx + 1

    def count(ph, n):
        lo = leftmost(ph, max(-32768, min(32767, phi1 - 2 * tol)))
        hv = phi1 + 2 * tol + 1
        hi = n if hv > 32767 else leftmost(ph, hv)
        return F32(min(hi - lo, 16))

    return np.array([np.sqrt(x1 * x1 + y1 * y1), z1, np.sqrt(best_d), best_z, best_t, np.sqrt(second_d),
                     np.sqrt(scatter[0]), np.sqrt(scatter[1]), count(pphi, pn), count(nphi, nn), min_dphi,
                     F32(phi1) * F32(3.0517578125e-05)], dtype=np.float32)


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
