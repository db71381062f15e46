"""The float64 training oracle (oracle/mlp_oracle.py) pinned by central finite differences: its
backpropagated gradients of the gated mean-squared loss equal the numerical derivative of its own
loss for sampled entries of every parameter tensor."""
import numpy as np

from oracle import mlp_oracle as mo


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    params = {name: rng.standard_normal(shape) * (0.5 / np.sqrt(shape[-1]) if len(shape) == 2 else 0.1)
              for name, shape in mo.SHAPES}
    n = 5
    stencil = rng.standard_normal((n, 384)) * 0.5
    particle = rng.uniform(0, 1, (n, 4))
    gate = np.array([0.0, 0.3, 1.0, 0.7, 1.0])
    target = rng.standard_normal((n, 3))
    _, grads = mo.loss_and_gradients(params, stencil, particle, gate, target)
    flat = mo.flatten(params)
    at, h = 0, 1e-6
    for name, shape in mo.SHAPES:
        size = int(np.prod(shape))
        for idx in rng.choice(size, size=min(6, size), replace=False):
            plus, minus = flat.copy(), flat.copy()
            plus[at + idx] += h
            minus[at + idx] -= h
            lp, _ = mo.loss_and_gradients(mo.unflatten(plus), stencil, particle, gate, target)
            lm, _ = mo.loss_and_gradients(mo.unflatten(minus), stencil, particle, gate, target)
            numeric = (lp - lm) / (2 * h)
            assert abs(numeric - grads[at + idx]) <= 1e-6 + 1e-5 * abs(numeric), (name, idx)
        at += size


def test_oracle_adam_first_step_moves_by_the_learning_rate():
    """With bias correction the first Adam step moves every parameter with a non-zero gradient by
    lr (up to eps), against the gradient's sign."""
    flat = np.zeros(4)
    grads = np.array([1e-3, -2.0, 5.0, 0.0])
    new, m, v = mo.adam(flat, grads, np.zeros(4), np.zeros(4), step=1, lr=0.01)
    assert np.allclose(new[:3], -0.01 * np.sign(grads[:3]), rtol=1e-4) and new[3] == 0.0


def test_bf16_rounding_matches_torch():
    """The oracle's bfloat16 rounding (nearest, ties to even) of the tensor-core operands."""
    import torch
    rng = np.random.default_rng(4)
    a = np.concatenate([rng.standard_normal(10000) * 10 ** rng.uniform(-6, 6, 10000),
                        1 + np.arange(256) * 2.0 ** -9, [0.0, -0.0, 1e-40, 3e38]])
    want = torch.tensor(a, dtype=torch.float32).bfloat16().double().numpy()
    assert np.array_equal(mo.bf16(a), want)
