"""Training of the advection surrogate on one-interval segments of the plain kernel.

Run on a CUDA device from the repository root:

    python -m wacommplusplus_b200.surrogate_train --out wacommplusplus_b200/surrogate_weights.npz

Segments: forward, deterministic intervals (dt = 30 s, explicit midpoint, FP32 step) of particles
placed uniformly over seeded synthetic forcing windows -- ROMS-shaped streamfunction flows
(``synthetic.RealisticForcing`` without land, several seeds and grid spacings) and uniform flows on
the analytic grid with random velocities -- a quarter of them released inside the interval.
Segments whose start or end is within two cells of the grid edge or at a vertical bound are
dropped (the surrogate hands those cases to the closures or to the plain kernel). Features and
targets follow ``surrogate.py``; the loss is the mean squared error of the scaled residual. The
network is trained by the library's own kernels (wacomm_b200_mlp_train_step: forward, loss,
backward and Adam in FP32 on the device); torch holds the data and the device buffers.
"""
import argparse
import math
import time

import numpy as np

from . import _native
from . import surrogate as sg
from . import synthetic as syn
from .engine import Engine
from .types import PARTICLE_DTYPE, default_config


def training_config():
    return default_config(random=False, dti=30.0, deltat=3600.0, integrator=2)


def training_windows(seed, n_realistic, n_uniform, frames):
    """(name, window) pairs: realistic flows then uniform flows."""
    rng = np.random.default_rng(seed)
    for n in range(n_realistic):
        spacing = [0.001, 0.0015, 0.002][n % 3]
        f = syn.RealisticForcing(eta=256, xi=256, s_rho=12, n_frames=frames, seed=1000 + seed * 97 + n,
                                 dlon=spacing, dlat=spacing, land_fraction=0.0, water_border=0)
        yield f"realistic{n}", f.window()
    for n in range(n_uniform):
        u, v = rng.uniform(-0.6, 0.6, 2)
        win = syn.config1_window(n_frames=2, u=float(u), v=float(v))
        win.w[:] = np.float32(rng.normal(0.0, 2e-4))
        yield f"uniform{n}", win


def segment_particles(rng, win, t, n):
    """n particles over the interior at interval t, a quarter released inside the interval."""
    out = np.zeros(n, dtype=PARTICLE_DTYPE)
    out["id"] = rng.integers(0, 2**62, n, dtype=np.uint64)
    out["j"] = rng.uniform(2.0, win.eta - 3.0, n)
    out["i"] = rng.uniform(2.0, win.xi - 3.0, n)
    out["k"] = -rng.uniform(0.02, win.sW - 2.02, n)
    out["health"] = 1.0
    t0, t1 = win.times[t], win.times[t + 1]
    late = rng.random(n) < 0.25
    out["time"] = np.where(late, rng.uniform(t0, t1, n), t0)
    return out


def targets(torch, win, t, start, end, cfg):
    """(stencil [n,384], particle [n,4], residual [n,3]) of finished segments, as torch tensors
    on the current device; rows follow `start`."""
    dev = torch.device("cuda")
    f64 = torch.float64
    T0, T1 = float(win.times[t]), float(win.times[t + 1])
    length = T1 - T0
    sW = win.sW
    j = torch.as_tensor(start["j"], device=dev)
    i = torch.as_tensor(start["i"], device=dev)
    k = torch.as_tensor(start["k"], device=dev)
    jI, iI, kI = torch.floor(j).long(), torch.floor(i).long(), torch.ceil(k).long()
    jF, iF, kF = j - jI, i - iI, kI - k
    a0 = ((torch.as_tensor(start["time"], device=dev) - T0) / length).clamp(min=0)
    fr = [torch.as_tensor(np.asarray(getattr(win, nm)[t + s]), device=dev)
          for s in (0, 1) for nm in ("u", "v", "w")]
    S = sg.stencil_features(*fr, jI, iI, kI)
    P = torch.stack([jF, iF, kF, a0], dim=1).float()
    amid = 0.5 * (a0 + 1)
    trem = (1 - a0) * length
    sRho = sW - 1
    ub = torch.zeros_like(j)
    vb = torch.zeros_like(j)
    wb = torch.zeros_like(j)
    for s, wt in ((0, 1 - amid), (1, amid)):
        u = fr[3 * s].double()
        v = fr[3 * s + 1].double()
        w = fr[3 * s + 2].double()
        ub += wt * sg._bilinear(u, kI + sRho - 1, jI, iI, jF, iF)
        vb += wt * sg._bilinear(v, kI + sRho - 1, jI, iI, jF, iF)
        wb += wt * ((1 - kF) * sg._bilinear(w, kI + sW - 1, jI, iI, jF, iF) +
                    kF * sg._bilinear(w, kI + sW - 2, jI, iI, jF, iF))
    h = torch.as_tensor(np.asarray(win.h), device=dev, dtype=f64)[None]
    z0 = torch.as_tensor(np.asarray(win.zeta[t]), device=dev, dtype=f64)[None]
    z1 = torch.as_tensor(np.asarray(win.zeta[t + 1]), device=dev, dtype=f64)[None]
    zero = torch.zeros_like(kI)
    hc = (sg._bilinear(h, zero, jI, iI, jF, iF) + (1 - amid) * sg._bilinear(z0, zero, jI, iI, jF, iF) +
          amid * sg._bilinear(z1, zero, jI, iI, jF, iF))
    xd, yd = (torch.as_tensor(a, device=dev) for a in sg.host_metric(win.lonRad, win.latRad))
    depth = torch.as_tensor(np.asarray(win.depthIntervals), device=dev)
    zdist = hc * depth[kI + sW - 2]
    dj = torch.as_tensor(end["j"], device=dev) - j
    di = torch.as_tensor(end["i"], device=dev) - i
    dk = torch.as_tensor(end["k"], device=dev) - k
    res = torch.stack([(di * xd[jI, iI] - ub * trem) / sg.OUT_SCALE[0],
                       (dj * yd[jI, iI] - vb * trem) / sg.OUT_SCALE[1],
                       (dk * zdist - (wb + cfg.sv) * trem) / sg.OUT_SCALE[2]], dim=1).float()
    return S, P, res


def generate(torch, engine, cfg, seed, n_realistic, n_uniform, frames, per_interval):
    rng = np.random.default_rng(seed)
    feats, parts, res = [], [], []
    kept = total = 0
    for name, win in training_windows(seed, n_realistic, n_uniform, frames):
        engine.load_window(win)
        for t in range(win.T - 1):
            start = segment_particles(rng, win, t, per_interval)
            engine.set_particles(start)
            engine.move_interval(t)
            end = engine.get_particles()
            kLower = -win.sW + 2
            ok = ((end["health"] > 0) & (end["j"] > 2) & (end["j"] < win.eta - 3) &
                  (end["i"] > 2) & (end["i"] < win.xi - 3) & (end["k"] < 0) & (end["k"] > kLower) &
                  (start["k"] > kLower + 0.01))
            total += len(start)
            kept += int(ok.sum())
            S, P, R = targets(torch, win, t, start[ok], end[ok], cfg)
            feats.append(S.to(torch.bfloat16))
            parts.append(P)
            res.append(R)
        print(f"  {name}: {kept}/{total} segments kept", flush=True)
    return torch.cat(feats), torch.cat(parts), torch.cat(res)


def initial_weights(seed):
    """He-style weights with zero biases and a small last layer: the correction starts near zero."""
    w = sg.random_weights(seed, scale=1.0)
    for k in ("b1", "b2", "b3", "b4"):
        w[k][:] = 0
    w["w4"] *= 0.1
    return w


class KernelTrainer:
    """Training of the MLP with the library's own kernels (wacomm_b200_mlp_train_step: forward,
    loss, backward and Adam on the device, the GEMMs of layers 1-3 and the weight gradients on the
    tensor cores in BF16 with FP32 accumulation); torch only holds the device buffers."""

    def __init__(self, torch, weights, batch):
        self.torch, self.lib, self.batch = torch, _native.lib(), batch
        flat = np.concatenate([np.asarray(weights[k], np.float32).reshape(-1)
                               for k, _ in sg.PARAMETERS])
        self.params = torch.tensor(flat, device="cuda")
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.work = torch.empty(self.lib.wacomm_b200_mlp_train_work_floats(batch),
                                dtype=torch.float32, device="cuda")
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.step = 0

    def run(self, S, P, G, R, lr=0.0, update=True):
        """One step on a batch of at most ``batch`` rows (float32 device tensors); returns the
        device loss of the batch (before the update)."""
        n = len(S)
        assert 0 < n <= self.batch
        S, P, G, R = (x.float().contiguous() for x in (S, P, G, R))
        if update:
            self.step += 1
        status = self.lib.wacomm_b200_mlp_train_step(
            S.data_ptr(), P.data_ptr(), G.data_ptr(), R.data_ptr(), n, self.params.data_ptr(),
            self.grads.data_ptr(), self.m.data_ptr(), self.v.data_ptr(), self.work.data_ptr(),
            self.loss.data_ptr(), max(self.step, 1), float(lr), int(update),
            self.torch.cuda.current_stream().cuda_stream)
        if status != 0:
            raise RuntimeError(f"wacomm_b200_mlp_train_step failed ({status})")
        return self.loss.clone()

    def error_flag(self):
        """Nonzero when a tensor-core GEMM of the steps so far gave up on a bounded wait (its
        results are then not valid); waits for the stream."""
        return int(self.work[:1].view(self.torch.int32).item())

    def weights(self):
        flat, out, at = self.params.cpu().numpy(), {}, 0
        for name, shape in sg.PARAMETERS:
            size = int(np.prod(shape))
            out[name] = flat[at:at + size].reshape(shape).copy()
            at += size
        return out

    def evaluate(self, S, P, G, R):
        """Mean loss over a set, in batches, without updating."""
        total = 0.0
        for c in range(0, len(S), self.batch):
            k = min(self.batch, len(S) - c)
            total += float(self.run(S[c:c + k], P[c:c + k], G[c:c + k], R[c:c + k],
                                    update=False)) * k
        return total / len(S)


def gates(torch, S):
    return torch.cat([sg.uniformity_gate(S[c:c + (1 << 20)].float()) for c in range(0, len(S), 1 << 20)])


def train(torch, S, P, R, epochs, batch, lr, seed):
    G = gates(torch, S)
    print(f"  gate: {float((G < 1).float().mean()):.3f} of segments below 1, "
          f"{float((G == 0).float().mean()):.3f} at 0", flush=True)
    trainer = KernelTrainer(torch, initial_weights(seed), batch)
    n = len(S)
    steps = epochs * (n // batch)
    hold = torch.randperm(n, device="cuda")[: min(n // 50, 200000)]
    mask = torch.ones(n, dtype=torch.bool, device="cuda")
    mask[hold] = False
    train_idx = torch.nonzero(mask).flatten()
    s = 0
    for epoch in range(epochs):
        perm = train_idx[torch.randperm(len(train_idx), device="cuda")]
        t0 = time.time()
        tot = torch.zeros(1, device="cuda")
        for b in range(len(perm) // batch):
            ix = perm[b * batch:(b + 1) * batch]
            rate = lr * 0.5 * (1 + math.cos(math.pi * min(s, steps) / steps))
            tot += trainer.run(S[ix], P[ix], G[ix], R[ix], rate)
            s += 1
        val = trainer.evaluate(S[hold], P[hold], G[hold], R[hold])
        base = torch.mean(R[hold].float() ** 2).item()
        print(f"  epoch {epoch}: train {float(tot) / max(1, len(perm) // batch):.4g} held-out "
              f"{val:.4g} (zero-residual baseline {base:.4g}) {time.time() - t0:.1f}s", flush=True)
    return trainer.weights()


def evaluate(weights, n_particles=32768, hours=24, seed=1, realistic=False):
    """Great-circle error (metres) after `hours` of the surrogate (PyTorch reference) against the
    reference-arithmetic kernel, on the analytic precision grid or on a realistic flow window
    without land; prints and returns the stats."""
    cfg = training_config()
    if realistic:
        win = syn.RealisticForcing(eta=256, xi=256, s_rho=12, n_frames=hours + 1, seed=4242,
                                   dlon=0.0015, dlat=0.0015, land_fraction=0.0,
                                   water_border=0).window()
        start = segment_particles(np.random.default_rng(seed), win, 0, n_particles)
        start["time"] = win.times[0]
    else:
        win = syn.config1_window(n_frames=hours + 1)
        start = syn.uniform_particles(n_particles, win.eta, win.xi, seed=seed, time=win.times[0])
    exact = Engine(0, arithmetic="reference")
    exact.set_config(cfg)
    exact.load_window(win)
    exact.set_particles(start)
    plain = Engine(0, arithmetic="fp32", storage="fp32")
    plain.set_config(cfg)
    plain.load_window(win)
    cur = start.copy()
    fallbacks = 0
    for t in range(hours):
        exact.move_interval(t)
        cur, fb = sg.reference_interval(weights, win, t, cur, cfg)
        if fb.any():
            fallbacks += int(fb.sum())
            plain.set_particles(cur[fb])
            plain.move_interval(t)
            cur[fb] = plain.get_particles()
    truth = exact.get_particles()
    exact.close()
    plain.close()
    err = sg.geo_error_m(win, cur, truth)
    stats = dict(mean=float(err.mean()), p99=float(np.quantile(err, 0.99)), max=float(err.max()),
                 fallbacks=fallbacks)
    print(f"{'realistic flow' if realistic else 'analytic grid'}, {hours} h, {n_particles} particles: "
          f"error mean {stats['mean']:.2f} m, "
          f"p99 {stats['p99']:.2f} m, max {stats['max']:.2f} m, fallback particle-intervals "
          f"{fallbacks}", flush=True)
    return stats


def time_steps(batch, steps=50):
    """Device time of the library's training step (forward, backward, Adam) on random data, and
    the rate of its tensor-core GEMMs (layers 1-3 forward, their weight gradients, the input
    gradients of layers 3 and 2)."""
    import torch
    rng = np.random.default_rng(0)
    S = torch.tensor(rng.standard_normal((batch, 384)).astype(np.float32) * 0.5, device="cuda")
    P = torch.rand(batch, 4, device="cuda")
    G = torch.rand(batch, device="cuda")
    R = torch.randn(batch, 3, device="cuda")
    trainer = KernelTrainer(torch, initial_weights(1), batch)
    for _ in range(5):
        trainer.run(S, P, G, R, lr=1e-4)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        trainer.run(S, P, G, R, lr=1e-4)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    flop = 2 * batch * (2 * 388 * 256 + 6 * 256 * 256)
    print(f"batch {batch}: {ms:.3f} ms per training step, {flop / ms / 1e9:.1f} TFLOP/s in the "
          f"tensor-core GEMMs, error flag {trainer.error_flag()}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=sg.DEFAULT_WEIGHTS)
    ap.add_argument("--realistic", type=int, default=6)
    ap.add_argument("--uniform", type=int, default=48)
    ap.add_argument("--frames", type=int, default=25)
    ap.add_argument("--per-interval", type=int, default=250000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--evaluate-only", action="store_true")
    ap.add_argument("--time-steps", type=int, default=0, metavar="BATCH",
                    help="time training steps of this batch on random data and exit")
    args = ap.parse_args()
    if args.time_steps:
        time_steps(args.time_steps)
        return
    if args.evaluate_only:
        evaluate(sg.load_weights(args.out))
        evaluate(sg.load_weights(args.out), realistic=True)
        return
    import torch
    cfg = training_config()
    engine = Engine(0, arithmetic="fp32", storage="fp32")
    engine.set_config(cfg)
    t0 = time.time()
    S, P, R = generate(torch, engine, cfg, args.seed, args.realistic, args.uniform, args.frames,
                       args.per_interval)
    engine.close()
    print(f"{len(S)} segments generated in {time.time() - t0:.1f}s; residual rms "
          f"{R.float().pow(2).mean(0).sqrt().tolist()}", flush=True)
    weights = train(torch, S, P, R, args.epochs, args.batch, args.lr, args.seed)
    sg.save_weights(args.out, weights, segments=len(S), epochs=args.epochs, seed=args.seed)
    print(f"weights written to {args.out}")
    evaluate(weights)
    evaluate(weights, realistic=True)


if __name__ == "__main__":
    main()
