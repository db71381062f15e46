"""Float64 restatement of the surrogate MLP's training step -- TEST INFRASTRUCTURE ONLY.

The checker of the library's training kernels (wacomm_b200_mlp_train_step): the same network
(388 -> 256 -> 256 -> 256 -> 3, GELU in its tanh form, outputs times the stencil's uniformity
gate), the mean-squared loss over batch x 3 outputs, its gradients by explicit backpropagation,
and Adam with the usual defaults (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected), all in
numpy float64. Parameters use the flat order w1, b1, w2, b2, w3, b3, w4, b4.
"""
import numpy as np

C0, C1 = 0.7978845608028654, 0.044715
SHAPES = (("w1", (256, 388)), ("b1", (256,)), ("w2", (256, 256)), ("b2", (256,)),
          ("w3", (256, 256)), ("b3", (256,)), ("w4", (3, 256)), ("b4", (3,)))


def unflatten(flat):
    out, at = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[at:at + n], np.float64).reshape(shape)
        at += n
    return out


def flatten(params):
    return np.concatenate([params[name].reshape(-1) for name, _ in SHAPES])


def _gelu(z):
    t = np.tanh(C0 * (z + C1 * z ** 3))
    return 0.5 * z * (1 + t), 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * C0 * (1 + 3 * C1 * z * z)


def bf16(a):
    """Round to bfloat16 (nearest, ties to even) through float32, as the tensor-core operands are
    rounded; returned as float64."""
    bits = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) >> 16 << 16
    return bits.astype(np.uint32).view(np.float32).astype(np.float64)


def loss_and_gradients(params, stencil, particle, gate, target, bf16_operands=False):
    """(loss, flat gradients) of one batch. With bf16_operands, the operands of the products the
    library computes on the tensor cores are rounded to bfloat16 first (layers 1-3 forward, their
    input and weight gradients, and the layer-4 weight gradient); the sums stay float64."""
    r = bf16 if bf16_operands else (lambda a: a)
    p = {k: np.asarray(v, np.float64) for k, v in params.items()}
    x = np.concatenate([stencil, particle], axis=1).astype(np.float64)
    g = np.asarray(gate, np.float64)[:, None]
    t = np.asarray(target, np.float64)
    z1 = r(x) @ r(p["w1"]).T + p["b1"]
    h1, d1 = _gelu(z1)
    z2 = r(h1) @ r(p["w2"]).T + p["b2"]
    h2, d2 = _gelu(z2)
    z3 = r(h2) @ r(p["w3"]).T + p["b3"]
    h3, d3 = _gelu(z3)
    o = h3 @ p["w4"].T + p["b4"]
    diff = o * g - t
    loss = float(np.mean(diff ** 2))
    do = 2 * diff * g / diff.size
    grads = {"w4": r(do).T @ r(h3), "b4": do.sum(0)}
    dz = (do @ p["w4"]) * d3
    grads["w3"], grads["b3"] = r(dz).T @ r(h2), dz.sum(0)
    dz = (r(dz) @ r(p["w3"])) * d2
    grads["w2"], grads["b2"] = r(dz).T @ r(h1), dz.sum(0)
    dz = (r(dz) @ r(p["w2"])) * d1
    grads["w1"], grads["b1"] = r(dz).T @ r(x), dz.sum(0)
    return loss, flatten(grads)


def adam(flat, grads, m, v, step, lr):
    """One Adam step of float64 copies; returns (params, m, v)."""
    m = 0.9 * m + 0.1 * grads
    v = 0.999 * v + 0.001 * grads * grads
    mh, vh = m / (1 - 0.9 ** step), v / (1 - 0.999 ** step)
    return flat - lr * mh / (np.sqrt(vh) + 1e-8), m, v
