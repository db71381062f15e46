"""Learned one-interval advection surrogate: definition, weights file and PyTorch FP32 reference.

The surrogate replaces the substep loop of a deterministic forward interval (Particle.cpp:178-814
with random off) by one evaluation of a small MLP per particle:

* inputs: the 4x4x4 stencil of u, v, w around the particle's cell and level at the two forcing
  records of the interval (384 values), plus the sub-cell offsets jF, iF, kF and the fraction of
  the interval already elapsed at activation (4 values);
* layers: 388 -> 256 -> 256 -> 256 -> 3, GELU (tanh form) between them;
* output: the correction, in metres, to the displacement that the velocity interpolated at the
  start position and the interval's mid time would give over the remaining time, scaled by a
  uniformity gate: min(1, sigma / GATE_SIGMA), sigma the RMS deviation of the stencil's u and v
  from their value at the cell's own corner (per record and field). In a spatially uniform flow
  the start-point displacement is exact and the gate makes the correction exactly zero.

The displacement is turned into grid units with the start cell's metric (host rules,
Particle.cpp:548-579), then the domain-edge closures are applied in closed form for the number of
substeps the interval has (reflection pins a particle against the edge exactly as repeated
reflectDomain calls do under a uniform per-substep displacement, NumericalHelpers.hpp:67-74),
and the vertical closures as at Particle.cpp:644-704. Particles the surrogate does not cover --
random walk on, backward tracking, drifting objects, a start outside the valid cells, a path
box that touches a dry node, a restart-clipped interval -- are flagged and moved by the plain
kernel instead.

This module holds the definition shared by training (``surrogate_train.py``), by the weights
upload of the engine and by the tests: the stencil order, the scales, the weights file layout and
``reference_interval``, a plain PyTorch FP32 implementation of the surrogate interval.
"""
import math
import os

import numpy as np

HIDDEN = 256
N_STENCIL = 384           # 2 records x 3 fields x 4 levels x 4 rows x 4 columns
N_PARTICLE = 4            # jF, iF, kF, activation fraction
N_INPUT = N_STENCIL + N_PARTICLE
N_OUTPUT = 3
U_SCALE = 1.0             # m/s per unit of the u, v features
W_SCALE = 1.0e-3          # m/s per unit of the w features
OUT_SCALE = (100.0, 100.0, 1.0)   # metres per unit of the three outputs (east, north, up)
GATE_SIGMA = 0.01         # m/s: stencil non-uniformity at which the correction is fully on
GATE_REF = (1 * 4 + 1) * 4 + 1    # position of the cell's own corner (level c=1, row a=1, column b=1) in a 64-block
EARTH_RADIUS = 6371000.0

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "surrogate_weights.npz")

# Order of the flat FP32 weight vector handed to wacomm_b200_set_surrogate.
PARAMETERS = (("w1", (HIDDEN, N_INPUT)), ("b1", (HIDDEN,)),
              ("w2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
              ("w3", (HIDDEN, HIDDEN)), ("b3", (HIDDEN,)),
              ("w4", (N_OUTPUT, HIDDEN)), ("b4", (N_OUTPUT,)))
N_PARAMETERS = sum(int(np.prod(shape)) for _, shape in PARAMETERS)


def flatten(weights):
    """The flat FP32 parameter vector (PARAMETERS order) of a name -> array mapping."""
    parts = []
    for name, shape in PARAMETERS:
        a = np.asarray(weights[name], dtype=np.float32)
        assert a.shape == shape, (name, a.shape, shape)
        parts.append(a.reshape(-1))
    return np.ascontiguousarray(np.concatenate(parts))


def unflatten(flat):
    out, at = {}, 0
    for name, shape in PARAMETERS:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[at:at + n], dtype=np.float32).reshape(shape)
        at += n
    return out


def load_weights(path=DEFAULT_WEIGHTS):
    with np.load(path) as data:
        return {name: data[name].astype(np.float32) for name, _ in PARAMETERS}


def save_weights(path, weights, **meta):
    np.savez(path, **{name: np.asarray(weights[name], np.float32) for name, _ in PARAMETERS},
             **{k: np.asarray(v) for k, v in meta.items()})


def random_weights(seed=0, scale=1.0):
    """Seeded weights of the right shapes (He-style), for kernel tests independent of training."""
    rng = np.random.default_rng(seed)
    out = {}
    for name, shape in PARAMETERS:
        if name.startswith("w"):
            out[name] = (rng.standard_normal(shape) * scale * math.sqrt(2.0 / shape[1])).astype(np.float32)
        else:
            out[name] = (0.1 * rng.standard_normal(shape)).astype(np.float32)
    return out


# ----------------------------------------------------------------------------- torch reference

def _torch():
    import torch
    return torch


def bf16_round(x):
    """Round a float32 tensor to bfloat16 and back (the kernel's operand precision)."""
    torch = _torch()
    return x.to(torch.bfloat16).to(torch.float32)


def gelu(x):
    """GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))."""
    torch = _torch()
    return 0.5 * x * (1.0 + torch.tanh(0.7978845608028654 * (x + 0.044715 * x * x * x)))


def host_metric(lon_rad, lat_rad):
    """(xdist, ydist) per cell in metres, host rules (Particle.cpp:548-574), as float64 arrays
    [eta][xi]; zero on the last row and column."""
    lon = np.asarray(lon_rad, np.float64)
    lat = np.asarray(lat_rad, np.float64)
    eta, xi = lon.shape
    x = np.zeros((eta, xi))
    y = np.zeros((eta, xi))
    s = np.sin(0.5 * (lat[1:, :-1] - lat[:-1, :-1]))
    d = s * s
    y[:-1, :-1] = 2.0 * np.arctan2(np.sqrt(d), np.sqrt(1.0 - d)) * EARTH_RADIUS
    s = np.sin(0.5 * (lon[:-1, 1:] - lon[:-1, :-1]))
    d = s * s * np.cos(lat[:-1, 1:]) * np.cos(lat[:-1, :-1])
    x[:-1, :-1] = 2.0 * np.arctan2(np.sqrt(d), np.sqrt(1.0 - d)) * EARTH_RADIUS
    return x, y


def stencil_features(u0, v0, w0, u1, v1, w1, jI, iI, kI):
    """[n, 384] float32 stencil features of cells (jI, iI) at levels kI.

    u*, v*: [sRho][eta][xi]; w*: [sW][eta][xi] tensors (storage level = logical level + levels - 1).
    Feature f = ((record * 3 + field) * 4 + c) * 16 + a * 4 + b is field (u, v, w) of record
    (t0, t1) at row clamp(jI - 1 + a), column clamp(iI - 1 + b) and level clamp(kI - 2 + c)
    (u, v on rho levels, w on w levels), scaled by 1/U_SCALE (u, v) and 1/W_SCALE (w)."""
    torch = _torch()
    sRho, eta, xi = u0.shape
    sW = w0.shape[0]
    dev = u0.device
    a = torch.arange(4, device=dev)
    rows = (jI[:, None] - 1 + a[None, :]).clamp(0, eta - 1)              # [n,4]
    cols = (iI[:, None] - 1 + a[None, :]).clamp(0, xi - 1)
    lev = kI[:, None] - 2 + a[None, :]                                    # [n,4]
    lr = lev.clamp(-sRho + 1, 0) + sRho - 1
    lw = lev.clamp(-sW + 1, 0) + sW - 1
    out = []
    for (fu, fv, fw) in ((u0, v0, w0), (u1, v1, w1)):
        for field, levels, scale in ((fu, lr, U_SCALE), (fv, lr, U_SCALE), (fw, lw, W_SCALE)):
            plane = field.shape[1] * field.shape[2]
            flat = field.reshape(-1)
            idx = (levels[:, :, None, None] * plane + rows[:, None, :, None] * xi +
                   cols[:, None, None, :])                                # [n,4(c),4(a),4(b)]
            out.append(flat[idx.reshape(idx.shape[0], -1)].to(torch.float32) / scale)
    return torch.cat(out, dim=1)


def uniformity_gate(stencil):
    """[n] gate in [0, 1] of stencil features [n, 384]: RMS over the u and v blocks of both records
    (features 0-127 and 192-319) of the deviation from each block's value at GATE_REF, in m/s,
    divided by GATE_SIGMA and capped at 1."""
    torch = _torch()
    blocks = [stencil[:, b * 64:(b + 1) * 64] for b in (0, 1, 3, 4)]
    total = sum(((x - x[:, GATE_REF:GATE_REF + 1]) ** 2).sum(1) for x in blocks)
    sigma = torch.sqrt(total / 256.0) * U_SCALE
    return torch.clamp(sigma / GATE_SIGMA, max=1.0)


def mlp(weights, stencil, particle, emulate_kernel=True):
    """[n, 3] outputs of the MLP from stencil [n, 384] and particle [n, 4] features.

    With emulate_kernel the operand roundings of the CUDA path are applied: stencil and the
    stencil part of w1 in bfloat16 (the per-cell GEMM), the per-cell partial sum in float16,
    hidden activations and w2, w3 in bfloat16; w4 and the particle part of w1 stay float32.
    The outputs are multiplied by the uniformity gate of the stencil."""
    torch = _torch()
    dev = stencil.device
    W = {k: torch.as_tensor(v, device=dev) for k, v in weights.items()}
    w1s, w1p = W["w1"][:, :N_STENCIL], W["w1"][:, N_STENCIL:]
    if emulate_kernel:
        z = bf16_round(stencil) @ bf16_round(w1s).T + W["b1"]
        z = z.to(torch.float16).to(torch.float32)
        h = bf16_round(gelu(z + particle @ w1p.T))
        h = bf16_round(gelu(h @ bf16_round(W["w2"]).T + W["b2"]))
        h = gelu(h @ bf16_round(W["w3"]).T + W["b3"])
        return (h @ W["w4"].T + W["b4"]) * uniformity_gate(stencil)[:, None]
    h = gelu(stencil @ w1s.T + particle @ w1p.T + W["b1"])
    h = gelu(h @ W["w2"].T + W["b2"])
    h = gelu(h @ W["w3"].T + W["b3"])
    return (h @ W["w4"].T + W["b4"]) * uniformity_gate(stencil)[:, None]


def _bilinear(field, level, jI, iI, jF, iF):
    """Bilinear value of field[level] at (jI + jF, iI + iF) with the reference corner weights."""
    plane = field.shape[1] * field.shape[2]
    xi = field.shape[2]
    flat = field.reshape(-1)
    base = level * plane + jI * xi + iI
    f00, f10 = flat[base], flat[base + xi]
    f11, f01 = flat[base + xi + 1], flat[base + 1]
    return (f00 * (1 - iF) * (1 - jF) + f10 * (1 - iF) * jF + f11 * iF * jF + f01 * iF * (1 - jF))


def geo_positions(window, records):
    """(lon, lat) degrees of records by bilinear interpolation of the window's lon/lat grid
    (the horizontal part of kji2deplatlon, OceanModelAdapter.cpp:271-310); NaN off the grid."""
    lon, lat = np.asarray(window.lon), np.asarray(window.lat)
    eta, xi = lon.shape
    j, i = records["j"], records["i"]
    jI = np.floor(j).astype(np.int64)
    iI = np.floor(i).astype(np.int64)
    ok = (jI >= 0) & (iI >= 0) & (jI + 1 < eta) & (iI + 1 < xi)
    jc, ic = np.where(ok, jI, 0), np.where(ok, iI, 0)
    jF, iF = j - jc, i - ic

    def bil(f):
        v = (f[jc, ic] * (1 - iF) * (1 - jF) + f[jc + 1, ic] * (1 - iF) * jF +
             f[jc + 1, ic + 1] * iF * jF + f[jc, ic + 1] * iF * (1 - jF))
        return np.where(ok, v, np.nan)
    return bil(lon), bil(lat)


def geo_error_m(window, a, b):
    """Great-circle distance in metres between the positions of records a and b."""
    lon1, lat1 = (np.radians(x) for x in geo_positions(window, a))
    lon2, lat2 = (np.radians(x) for x in geo_positions(window, b))
    s = (np.sin(0.5 * (lat2 - lat1)) ** 2 +
         np.cos(lat1) * np.cos(lat2) * np.sin(0.5 * (lon2 - lon1)) ** 2)
    return 2 * EARTH_RADIUS * np.arcsin(np.sqrt(np.clip(s, 0, 1)))


def pinned_axis(x0, disp, n_sub, maximum, closure):
    """Closed-form end of n_sub equal substeps of `disp`/n_sub along one axis that may leave
    [0, maximum): returns (x, crossed_step) where crossed_step is the 1-based substep of the first
    exit (n_sub + 1 when none). Reflection alternates the overshoot like repeated reflectDomain;
    constraint and kill are resolved by the caller from crossed_step."""
    torch = _torch()
    d = disp / n_sub
    end = x0 + disp
    big = n_sub + 1
    up = end >= maximum
    down = end < 0
    m_up = torch.where(d > 0, torch.floor((maximum - x0) / torch.where(d > 0, d, 1.0)) + 1, big)
    m_dn = torch.where(d < 0, torch.floor(x0 / torch.where(d < 0, -d, 1.0)) + 1, big)
    m = torch.minimum(torch.where(up, m_up, torch.where(down, m_dn, big)), big)
    r = n_sub - m
    e_up = x0 + m * d - maximum
    e_dn = -(x0 + m * d)
    ad = d.abs()
    e = torch.where(up, e_up, e_dn).clamp(min=0)
    e = torch.where(torch.remainder(r, 2) == 0, e, ad - e).clamp(min=0)
    pinned = torch.where(up, maximum - e, e).clamp(0.0, math.nextafter(maximum, 0.0))
    x = torch.where(up | down, pinned, end)
    return x, torch.where(up | down, m, big)


def reference_interval(weights, window, t, particles, cfg, emulate_kernel=True):
    """One forward, deterministic interval [times[t], times[t+1]] of every particle by the
    surrogate, in float64 bookkeeping around the float32 MLP. Returns (records, fallback) where
    fallback marks the particles the surrogate leaves to the plain kernel (unchanged here).

    ``window`` holds float32 arrays u, v, w, zeta [T][...], h, lonRad, latRad, depthIntervals,
    mask; ``particles`` is a PARTICLE_DTYPE array; ``cfg`` a config_data."""
    torch = _torch()
    dev = torch.device("cpu")
    f64 = torch.float64
    rec = particles.copy()
    n = len(rec)
    T0, T1 = float(window.times[t]), float(window.times[t + 1])
    length = T1 - T0
    eta, xi = window.h.shape
    sW = len(window.depthIntervals) + 1
    kLower = -sW + 2
    j = torch.as_tensor(rec["j"], dtype=f64)
    i = torch.as_tensor(rec["i"], dtype=f64)
    k = torch.as_tensor(rec["k"], dtype=f64)
    rel = torch.as_tensor(rec["time"], dtype=f64)
    age = torch.as_tensor(rec["age"], dtype=f64)
    health = torch.as_tensor(rec["health"], dtype=f64)
    ptype = torch.as_tensor(rec["driftObjectType"].astype(np.int64))

    active = (health > 0) & (rel < T1)                      # released before the interval ends
    alpha0 = ((rel - T0) / length).clamp(min=0.0)
    jI = torch.floor(j).to(torch.int64)
    iI = torch.floor(i).to(torch.int64)
    kI = torch.ceil(k).to(torch.int64)
    jF, iF, kF = j - jI, i - iI, kI - k
    valid = (jI >= 0) & (iI >= 0) & (jI + 1 < eta) & (iI + 1 < xi) & (kI <= 0) & (kI >= kLower)
    fallback = active & ~valid
    if cfg.random or cfg.trackingDirection < 0 or math.isfinite(cfg.restartCheckpoint):
        fallback = active.clone()
    if cfg.driftModel == 1:
        fallback |= active & (ptype != 0)
    fallback |= active & (health < cfg.survprob)
    run = active & ~fallback
    idx = torch.nonzero(run).flatten()
    if len(idx) == 0:
        return rec, fallback.numpy()
    jI_, iI_, kI_ = jI[idx], iI[idx], kI[idx]
    frames = [torch.as_tensor(np.asarray(getattr(window, name)[t + s]), dtype=torch.float32)
              for s in (0, 1) for name in ("u", "v", "w")]
    S = stencil_features(frames[0], frames[1], frames[2], frames[3], frames[4], frames[5],
                         jI_, iI_, kI_)
    P = torch.stack([jF[idx], iF[idx], kF[idx], alpha0[idx]], dim=1).to(torch.float32)
    y = mlp(weights, S, P, emulate_kernel).to(f64)

    a0 = alpha0[idx]
    amid = 0.5 * (a0 + 1.0)
    trem = (1.0 - a0) * length
    sRho = sW - 1
    lr = kI_ + sRho - 1
    jf, if_ = jF[idx], iF[idx]
    ub = torch.zeros(len(idx), dtype=f64)
    vb = torch.zeros(len(idx), dtype=f64)
    wb = torch.zeros(len(idx), dtype=f64)
    for s, weight in ((0, 1.0 - amid), (1, amid)):
        u = torch.as_tensor(np.asarray(window.u[t + s]), dtype=f64)
        v = torch.as_tensor(np.asarray(window.v[t + s]), dtype=f64)
        w = torch.as_tensor(np.asarray(window.w[t + s]), dtype=f64)
        ub += weight * _bilinear(u, lr, jI_, iI_, jf, if_)
        vb += weight * _bilinear(v, lr, jI_, iI_, jf, if_)
        kf = kF[idx]
        wb += weight * ((1 - kf) * _bilinear(w, kI_ + sW - 1, jI_, iI_, jf, if_) +
                        kf * _bilinear(w, kI_ + sW - 2, jI_, iI_, jf, if_))
    h = torch.as_tensor(np.asarray(window.h), dtype=f64)[None]
    z0 = torch.as_tensor(np.asarray(window.zeta[t]), dtype=f64)[None]
    z1 = torch.as_tensor(np.asarray(window.zeta[t + 1]), dtype=f64)[None]
    zero = torch.zeros_like(kI_)
    hc = (_bilinear(h, zero, jI_, iI_, jf, if_) +
          (1 - amid) * _bilinear(z0, zero, jI_, iI_, jf, if_) + amid * _bilinear(z1, zero, jI_, iI_, jf, if_))
    xdist, ydist = (torch.as_tensor(a, dtype=f64) for a in host_metric(window.lonRad, window.latRad))
    xd = xdist[jI_, iI_]
    yd = ydist[jI_, iI_]
    depth = torch.as_tensor(np.asarray(window.depthIntervals), dtype=f64)
    zdist = hc * depth[kI_ + sW - 2]
    de = ub * trem + OUT_SCALE[0] * y[:, 0]
    dn = vb * trem + OUT_SCALE[1] * y[:, 1]
    du = (wb + cfg.sv) * trem + OUT_SCALE[2] * y[:, 2]
    n_sub = torch.ceil(trem / cfg.dti - 1e-9).clamp(min=1)
    dI, dJ, dK = de / xd, dn / yd, du / zdist

    j0, i0, k0 = j[idx], i[idx], k[idx]
    jn, mj = pinned_axis(j0, dJ, n_sub, float(eta - 1), cfg.horizontalClosure)
    inew, mi = pinned_axis(i0, dI, n_sub, float(xi - 1), cfg.horizontalClosure)
    crossed = torch.minimum(mj, mi) <= n_sub
    dead = torch.zeros(len(idx), dtype=torch.bool)
    if cfg.horizontalClosure == 1:      # constraint: stays at the last in-domain substep
        m = torch.minimum(mj, mi)
        keep = (m - 1) / n_sub
        jn = torch.where(crossed, j0 + keep * dJ, j0 + dJ)
        inew = torch.where(crossed, i0 + keep * dI, i0 + dI)
    elif cfg.horizontalClosure == 2:    # kill
        dead |= crossed
        jn = torch.where(crossed, j0, jn)
        inew = torch.where(crossed, i0, inew)
    kn = k0 + dK
    up = kn > 0
    if cfg.upperClosure == 1:
        kn = torch.where(up, torch.zeros_like(kn), kn)
    elif cfg.upperClosure == 2:
        dead |= up
    elif cfg.upperClosure == 3:
        kn = torch.where(up, -kn, kn)
    lo = kn < kLower
    if cfg.lowerClosure == 1:
        kn = torch.where(lo, torch.full_like(kn, float(kLower)), kn)
    elif cfg.lowerClosure == 2:
        dead |= lo
    elif cfg.lowerClosure == 3:
        kn = torch.where(lo, 2.0 * kLower - kn, kn)

    # dry nodes inside the path box (one node of margin) -> plain kernel
    mask = np.asarray(window.mask) if getattr(window, "mask", None) is not None else np.ones((eta, xi))
    dry = (mask == 0) | (np.asarray(window.h) <= cfg.shoreLimit)
    pre = np.zeros((eta + 1, xi + 1), np.int64)
    pre[1:, 1:] = np.cumsum(np.cumsum(dry, 0), 1)
    pre = torch.as_tensor(pre)
    ja = torch.minimum(j0, jn).floor().to(torch.int64).clamp(0, eta - 1)
    jb = (torch.maximum(j0, jn).floor().to(torch.int64) + 1).clamp(0, eta - 1)
    ia = torch.minimum(i0, inew).floor().to(torch.int64).clamp(0, xi - 1)
    ib = (torch.maximum(i0, inew).floor().to(torch.int64) + 1).clamp(0, xi - 1)
    dry_count = pre[jb + 1, ib + 1] - pre[ja, ib + 1] - pre[jb + 1, ia] + pre[ja, ia]
    wet = dry_count == 0
    new_age = age[idx] + trem
    new_health = torch.exp(-new_age / cfg.tau0)
    dead = dead | (new_health < cfg.survprob)
    done = idx[wet]
    fallback[idx[~wet]] = True
    rec_j, rec_i, rec_k = rec["j"], rec["i"], rec["k"]
    rec_j[done.numpy()] = jn[wet].numpy()
    rec_i[done.numpy()] = inew[wet].numpy()
    rec_k[done.numpy()] = kn[wet].numpy()
    rec["age"][done.numpy()] = new_age[wet].numpy()
    rec["health"][done.numpy()] = torch.where(dead[wet], torch.full_like(new_health[wet], -1.0),
                                              new_health[wet]).numpy()
    return rec, fallback.numpy()
