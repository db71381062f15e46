"""The surrogate's definition on the CPU: weights file, gate, closed-form edge closures, and the
PyTorch reference on uniform flow (where the start-point displacement is exact)."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from wacommplusplus_b200 import surrogate as sg
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.types import default_config


def test_shipped_weights_have_the_declared_layout():
    w = sg.load_weights()
    assert set(w) == {name for name, _ in sg.PARAMETERS}
    for name, shape in sg.PARAMETERS:
        assert w[name].shape == shape and w[name].dtype == np.float32
        assert np.all(np.isfinite(w[name]))
    flat = sg.flatten(w)
    assert flat.shape == (sg.N_PARAMETERS,) == (231939,)
    back = sg.unflatten(flat)
    assert all(np.array_equal(back[k], w[k]) for k in w)


def test_gate_is_zero_on_uniform_flow_and_one_on_sheared_flow():
    win = syn.config1_window(n_frames=2)
    fr = [torch.tensor(np.asarray(getattr(win, n)[s])) for s in (0, 1) for n in ("u", "v", "w")]
    jI = torch.tensor([5, 60, 120])
    iI = torch.tensor([7, 64, 3])
    kI = torch.tensor([0, -3, -8])
    S = sg.stencil_features(*fr, jI, iI, kI)
    assert S.shape == (3, 384)
    assert torch.all(sg.uniformity_gate(S) == 0)
    # u of record 0 at the four levels of the first rows and columns of the stencil
    assert torch.allclose(S[:, 0:64], torch.full((3, 64), 0.2))
    assert torch.allclose(S[:, 64:128], torch.full((3, 64), 0.1))
    fr[0] = fr[0] + 0.05 * torch.arange(win.xi, dtype=torch.float32)[None, None, :]
    S = sg.stencil_features(*fr, jI, iI, kI)
    assert torch.all(sg.uniformity_gate(S) == 1)


@pytest.mark.parametrize("seed", range(6))
def test_pinned_axis_matches_repeated_reflection(seed):
    """Closed-form reflection at the domain edge against the reference's per-substep
    reflectDomain (NumericalHelpers.hpp:67-74) under a uniform per-substep displacement."""
    rng = np.random.default_rng(seed)
    maximum = 127.0
    x0 = torch.tensor(rng.uniform(0.5, 126.5, 400), dtype=torch.float64)
    disp = torch.tensor(rng.uniform(-30, 30, 400), dtype=torch.float64)
    n = torch.full((400,), 120.0, dtype=torch.float64)
    got, _ = sg.pinned_axis(x0, disp, n, maximum, 3)

    def reflect(c):
        r = math.fmod(c, 2 * maximum)
        if r < 0:
            r += 2 * maximum
        if r >= maximum:
            r = 2 * maximum - r
        if r >= maximum:
            r = math.nextafter(maximum, 0)
        return r

    for a, d, g in zip(x0.tolist(), disp.tolist(), got.tolist()):
        x = a
        step = d / 120
        for _ in range(120):
            c = x + step
            x = reflect(c) if (c >= maximum or c < 0) else c
        assert abs(x - g) < 1e-9 * max(1.0, abs(step)) + 1e-9, (a, d, x, g)


def test_reference_interval_is_the_exact_displacement_on_uniform_flow():
    win = syn.config1_window(n_frames=2)
    cfg = default_config(random=False)
    p = syn.uniform_particles(500, win.eta, win.xi, time=win.times[0])
    p["j"] = np.clip(p["j"], 2, 100)
    p["i"] = np.clip(p["i"], 2, 100)
    out, fb = sg.reference_interval(sg.load_weights(), win, 0, p, cfg)
    assert not fb.any()
    xd, yd = sg.host_metric(win.lonRad, win.latRad)
    jI, iI = np.floor(p["j"]).astype(int), np.floor(p["i"]).astype(int)
    u, v = float(np.float32(0.2)), float(np.float32(0.1))   # the forcing is stored in float32
    assert np.allclose(out["i"] - p["i"], u * 3600 / xd[jI, iI], rtol=0, atol=1e-9)
    assert np.allclose(out["j"] - p["j"], v * 3600 / yd[jI, iI], rtol=0, atol=1e-9)
    assert np.array_equal(out["k"], p["k"])
    assert np.allclose(out["age"], 3600.0)
    assert np.allclose(out["health"], np.exp(-3600.0 / cfg.tau0))
