"""Training of the surrogate MLP with the library's own kernels (wacomm_b200_mlp_train_step: BF16
tcgen05 GEMMs for layers 1-3 and the weight gradients, FP32 elsewhere): gradients and the Adam
step against the float64 oracle (oracle/mlp_oracle.py), and what the trained network gains over
the method without it on held-out segments of the plain kernel."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo
from wacommplusplus_b200 import surrogate as sg

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    stencil = (rng.standard_normal((n, 384)) * 0.5).astype(np.float32)
    particle = rng.uniform(0, 1, (n, 4)).astype(np.float32)
    gate = rng.uniform(0, 1, n).astype(np.float32)
    gate[::7], gate[1::7] = 0.0, 1.0
    target = rng.standard_normal((n, 3)).astype(np.float32)
    return stencil, particle, gate, target


def _cuda(*arrays):
    return [torch.tensor(a, device="cuda") for a in arrays]


@pytest.mark.parametrize("n", [37, 300, 5000])
def test_gradients_match_the_oracle(cuda_device, n):
    """The training GEMMs run on the tensor cores with BF16 operands and FP32 accumulation. Against
    the float64 backpropagation that rounds the same operands to BF16 (mlp_oracle, bf16_operands)
    the gradients agree to 2e-3 of each tensor's largest entry (FP32 sums, and a BF16 rounding
    that the kernel's FP32 activation and the oracle's float64 one may take to different sides);
    against the unrounded float64 gradients, to 5e-2 (the BF16 roundings themselves)."""
    from wacommplusplus_b200.surrogate_train import KernelTrainer
    weights = sg.random_weights(seed=5)
    data = _batch(n, seed=n)
    trainer = KernelTrainer(torch, weights, batch=max(512, n))
    loss = float(trainer.run(*_cuda(*data), update=False))
    assert trainer.error_flag() == 0
    want_loss, want = mo.loss_and_gradients(weights, *data, bf16_operands=True)
    exact_loss, exact = mo.loss_and_gradients(weights, *data)
    got = trainer.grads.cpu().numpy().astype(np.float64)
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss), (loss, want_loss)
    assert abs(loss - exact_loss) <= 1e-2 * abs(exact_loss), (loss, exact_loss)
    at = 0
    for name, shape in mo.SHAPES:
        size = int(np.prod(shape))
        g, w, x = got[at:at + size], want[at:at + size], exact[at:at + size]
        rel = np.abs(g - w).max() / max(np.abs(w).max(), 1e-30)
        assert rel < 2e-3, (name, rel)
        rel = np.abs(g - x).max() / max(np.abs(x).max(), 1e-30)
        assert rel < 5e-2, (name, rel)
        at += size


def test_weight_gradients_are_reproducible(cuda_device):
    """The weight gradients reduce the batch in a fixed order (per-split partial sums, summed in
    order): two runs of the same batch give the same bits."""
    from wacommplusplus_b200.surrogate_train import KernelTrainer
    data = _cuda(*_batch(20000, seed=3))
    first = KernelTrainer(torch, sg.random_weights(seed=2), batch=20000)
    first.run(*data, update=False)
    second = KernelTrainer(torch, sg.random_weights(seed=2), batch=20000)
    second.run(*data, update=False)
    assert torch.equal(first.grads, second.grads)


def test_adam_steps_match_the_oracle(cuda_device):
    from wacommplusplus_b200.surrogate_train import KernelTrainer
    weights = sg.random_weights(seed=6)
    trainer = KernelTrainer(torch, weights, batch=128)
    flat = mo.flatten({k: np.asarray(v, np.float64) for k, v in weights.items()})
    m = np.zeros_like(flat)
    v = np.zeros_like(flat)
    for step, lr in ((1, 1e-3), (2, 5e-4)):
        data = _batch(128, seed=10 + step)
        trainer.run(*_cuda(*data), lr=lr, update=True)
        grads = trainer.grads.cpu().numpy().astype(np.float64)  # the step's own gradients
        flat, m, v = mo.adam(flat, grads, m, v, step, lr)
        got = trainer.params.cpu().numpy().astype(np.float64)
        assert np.abs(got - flat).max() <= 1e-6 * max(1.0, np.abs(flat).max()), step


def test_trained_network_gains_over_the_method_without_it(cuda_device):
    """Held-out one-hour segments of the plain kernel on a streamfunction flow the training never
    saw (a new seed): the surrogate's residual error with the shipped network against the
    start-point displacement alone (zero correction), and a short run of the library's training
    kernels from the initial weights on these segments lowers the loss."""
    from wacommplusplus_b200.engine import Engine
    from wacommplusplus_b200 import surrogate_train as st
    cfg = st.training_config()
    with Engine(cuda_device, arithmetic="fp32", storage="fp32") as e:
        e.set_config(cfg)
        S, P, R = st.generate(torch, e, cfg, seed=91, n_realistic=1, n_uniform=0, frames=4,
                              per_interval=60000)
    G = st.gates(torch, S)
    zero = float(torch.mean(R.float() ** 2))
    trained = st.KernelTrainer(torch, sg.load_weights(), batch=16384).evaluate(S, P, G, R)
    print(f"\nheld-out segments: {len(S)}; mean squared residual, zero correction {zero:.4g}, "
          f"shipped network {trained:.4g}")
    assert trained < 0.3 * zero
    fresh = st.KernelTrainer(torch, st.initial_weights(3), batch=4096)
    before = fresh.evaluate(S, P, G, R)
    for step in range(300):
        ix = torch.randint(0, len(S), (4096,), device="cuda")
        fresh.run(S[ix], P[ix], G[ix], R[ix], lr=1e-3)
    after = fresh.evaluate(S, P, G, R)
    print(f"own-kernel training, 300 steps: {before:.4g} -> {after:.4g}")
    assert after < 0.5 * before
