"""CPU restatement (numpy) of the learned proposal network of
gjxl_b200/csrc/cnn.cu: forward pass, loss, backward pass and AdamW.

TEST INFRASTRUCTURE ONLY: the checker of the device training kernels'
gradients. The reference has no learned component; this file restates the
network this repository defines, so it is pinned by its own finite-difference
check (tests/test_cnn_cpu.py) rather than by reference outputs.

With bf16=True, weights and activations are rounded to BF16 (round to
nearest even) exactly where the device rounds them, products accumulate in
FP32, and the backward pass treats the roundings as the identity, as the
device does. With bf16=False everything is float64, for finite differences.
"""

from __future__ import annotations

import numpy as np

IN, IN_C, C, STRATEGIES, HEAD = 80, 4, 32, 27, 28
# (cin, in_size, out_size, stride) of the four convolutions.
LAYERS = [(IN_C, 80, 40, 2), (C, 40, 20, 2), (C, 20, 10, 2), (C, 10, 10, 1)]


def param_layout() -> list[tuple[str, int, tuple]]:
    """(name, offset, shape) of every parameter block, in the device layout."""
    out, offset = [], 0
    for i, (cin, _, _, _) in enumerate(LAYERS):
        shape = (C, 3, 3, cin)
        out.append((f"w{i + 1}", offset, shape))
        offset += int(np.prod(shape))
        out.append((f"b{i + 1}", offset, (C,)))
        offset += C
    out.append(("wh", offset, (HEAD, C)))
    offset += HEAD * C
    out.append(("bh", offset, (HEAD,)))
    return out


PARAMS = sum(int(np.prod(shape)) for _, _, shape in param_layout())


def unpack(flat: np.ndarray) -> dict[str, np.ndarray]:
    return {name: flat[offset:offset + int(np.prod(shape))].reshape(shape)
            for name, offset, shape in param_layout()}


def round_bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even)."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation (FP32)."""
    rng = np.random.default_rng(seed)
    flat = np.zeros(PARAMS, np.float32)
    for name, offset, shape in param_layout():
        n = int(np.prod(shape))
        if name.startswith("w"):
            fan_in = int(np.prod(shape[1:]))
            flat[offset:offset + n] = rng.normal(0, np.sqrt(2.0 / fan_in), n)
    return flat


def _patches(x: np.ndarray, out_size: int, stride: int) -> np.ndarray:
    """[N, out, out, 9 * cin] patches in (ky, kx, ci) order, zero padding 1."""
    n, size, _, cin = x.shape
    xp = np.zeros((n, size + 2, size + 2, cin), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = []
    for ky in range(3):
        for kx in range(3):
            cols.append(xp[:, ky:ky + stride * out_size:stride, kx:kx + stride * out_size:stride])
    return np.concatenate(cols, axis=-1)


def forward(flat: np.ndarray, x0: np.ndarray, bf16: bool = True) -> dict:
    """x0: [N, 80, 80, 4] inputs (BF16 values when bf16). Returns the
    activations (conv outputs after ReLU) and the head [N, 64, 28]."""
    p = unpack(flat.astype(np.float32 if bf16 else np.float64))
    rnd = round_bf16 if bf16 else (lambda a: a)
    acts = [x0]
    x = x0
    for i, (cin, _, out_size, stride) in enumerate(LAYERS):
        w = rnd(p[f"w{i + 1}"]).reshape(C, 9 * cin)
        z = _patches(x, out_size, stride) @ w.T + p[f"b{i + 1}"]
        x = rnd(np.maximum(z, 0))
        acts.append(x)
    centre = x[:, 1:9, 1:9, :].reshape(x.shape[0], 64, C)
    head = centre @ rnd(p["wh"]).T + p["bh"]
    return {"acts": acts, "head": head}


def loss_and_grad(head: np.ndarray, labels: np.ndarray, targets: np.ndarray,
                  weights: np.ndarray, qf_weight: float) -> tuple[float, np.ndarray]:
    """Mean over all N * 64 block slots of w * (CE + qf_weight * e^2)."""
    n = head.shape[0]
    logits = head[..., :STRATEGIES]
    m = logits.max(-1, keepdims=True)
    lse = m[..., 0] + np.log(np.exp(logits - m).sum(-1))
    picked = np.take_along_axis(logits, labels[..., None].astype(np.int64), -1)[..., 0]
    e = head[..., STRATEGIES] - targets
    loss = float((weights * ((lse - picked) + qf_weight * e * e)).sum() / (n * 64))
    scale = (weights / (n * 64))[..., None]
    d = np.zeros_like(head)
    soft = np.exp(logits - lse[..., None])
    onehot = np.zeros_like(soft)
    np.put_along_axis(onehot, labels[..., None].astype(np.int64), 1.0, -1)
    d[..., :STRATEGIES] = scale * (soft - onehot)
    d[..., STRATEGIES] = scale[..., 0] * 2.0 * qf_weight * e
    return loss, d


def backward(flat: np.ndarray, fwd: dict, dhead: np.ndarray, bf16: bool = True) -> np.ndarray:
    """Gradient of the loss with respect to the flat parameters."""
    p = unpack(flat.astype(np.float32 if bf16 else np.float64))
    rnd = round_bf16 if bf16 else (lambda a: a)
    grads = {}
    acts = fwd["acts"]
    n = dhead.shape[0]
    a4 = acts[4]
    centre = a4[:, 1:9, 1:9, :].reshape(n, 64, C)
    grads["wh"] = np.einsum("nik,nic->kc", dhead, centre)
    grads["bh"] = dhead.sum((0, 1))
    dy = np.zeros_like(a4)
    dy[:, 1:9, 1:9, :] = (dhead @ rnd(p["wh"])).reshape(n, 8, 8, C)
    for i in range(3, -1, -1):
        cin, in_size, out_size, stride = LAYERS[i]
        y = acts[i + 1]
        dz = dy * (y > 0)
        patches = _patches(acts[i], out_size, stride)
        dzf = dz.reshape(-1, C)
        grads[f"w{i + 1}"] = (dzf.T @ patches.reshape(-1, 9 * cin)).reshape(C, 3, 3, cin)
        grads[f"b{i + 1}"] = dzf.sum(0)
        if i > 0:
            w = rnd(p[f"w{i + 1}"]).reshape(C, 9 * cin)
            dpatch = (dz @ w).reshape(n, out_size, out_size, 3, 3, cin)
            dxp = np.zeros((n, in_size + 2, in_size + 2, cin), dz.dtype)
            for ky in range(3):
                for kx in range(3):
                    dxp[:, ky:ky + stride * out_size:stride,
                        kx:kx + stride * out_size:stride] += dpatch[:, :, :, ky, kx]
            dy = dxp[:, 1:-1, 1:-1]
    out = np.zeros(PARAMS, np.float64)
    for name, offset, shape in param_layout():
        out[offset:offset + int(np.prod(shape))] = grads[name].reshape(-1)
    return out


def adamw(params, grads, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
    """One AdamW step (decoupled weight decay), in float32 like the device."""
    params, grads = params.astype(np.float32), grads.astype(np.float32)
    m = (beta1 * m + (1 - beta1) * grads).astype(np.float32)
    v = (beta2 * v + (1 - beta2) * grads * grads).astype(np.float32)
    mhat = m / np.float32(1 - beta1 ** step)
    vhat = v / np.float32(1 - beta2 ** step)
    params = params - np.float32(lr) * (mhat / (np.sqrt(vhat) + np.float32(eps)) +
                                        np.float32(weight_decay) * params)
    return params.astype(np.float32), m, v
