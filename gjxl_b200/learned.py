"""The learned proposal network (gjxl_b200_cnn_*): training on the plain
search's decisions, the committed weights, and the learned-versus-plain
measurement.

Training examples come from the plain analysis itself: for every 64x64 tile
of a seeded synthetic image analysed at distance d, the network's input is
the tile of Gaborish-inverted XYB the search saw (with an 8-px halo and
log2 d), and its targets per 8x8 block are the strategy the greedy merge
chose (the code of the transform covering the block) and log(final field /
adjusted field), the correction the refinement loop applied to the field it
started from. Training runs the library's own forward, backward and AdamW
kernels; torch holds the device memory only.

    python -m gjxl_b200.learned train --images 128 --size 1024 --out weights.f32
"""

from __future__ import annotations

import argparse
import ctypes
import json
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .session import AnalysisSession

# Trained parameters shipped with the package (FP32, the device layout).
WEIGHTS_PATH = Path(__file__).resolve().parent / "learned_proposals.f32"
DISTANCES = (0.5, 1.0, 2.0, 3.0)
QF_WEIGHT = 4.0


class _CudaArray:
    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def device_array(ptr: int, shape, dtype) -> torch.Tensor:
    """Torch view (no copy) of device memory the library owns."""
    return torch.as_tensor(_CudaArray(ptr, shape, np.dtype(dtype).str), device="cuda")


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def param_count() -> int:
    return int(_lib.load().gjxl_b200_cnn_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He initialisation of the convolutions and head; zero biases."""
    rng = np.random.default_rng(seed)
    flat = np.zeros(param_count(), np.float32)
    offset = 0
    for cin in (4, 32, 32, 32):
        n = 32 * 9 * cin
        flat[offset:offset + n] = rng.normal(0, np.sqrt(2.0 / (9 * cin)), n)
        offset += n + 32
    flat[offset:offset + 28 * 32] = rng.normal(0, np.sqrt(1.0 / 32), 28 * 32)
    return flat


class ProposalNetwork:
    """Parameters and AdamW state on the device, and one workspace."""

    def __init__(self, flat: np.ndarray | None = None, seed: int = 0):
        flat = init_params(seed) if flat is None else np.asarray(flat, np.float32)
        assert flat.size == param_count()
        self.params = torch.from_numpy(flat.copy()).cuda()
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self._tiles = 0
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")

    @classmethod
    def load(cls, path: Path = WEIGHTS_PATH) -> "ProposalNetwork":
        return cls(np.fromfile(path, dtype=np.float32))

    def save(self, path: Path) -> None:
        self.params.cpu().numpy().astype(np.float32).tofile(path)

    def ensure(self, tiles: int) -> None:
        if tiles > self._tiles:
            lib = _lib.load()
            self.workspace = torch.empty(lib.gjxl_b200_cnn_workspace_bytes(tiles),
                                         dtype=torch.uint8, device="cuda")
            self.scratch = torch.empty(lib.gjxl_b200_cnn_train_scratch_bytes(tiles),
                                       dtype=torch.uint8, device="cuda")
            self._tiles = tiles

    def inputs(self, tiles: int) -> torch.Tensor:
        """The workspace's input tiles, [tiles, 80, 80, 4] raw BF16 bits."""
        return self.workspace[:tiles * 80 * 80 * 4 * 2].view(torch.int16).view(tiles, 80, 80, 4)

    def gather(self, opsin_ptr: int, stride: int, pitch: int, pw: int, ph: int, tiles: int,
               distance: float) -> None:
        self.ensure(tiles)
        _lib.call("gjxl_b200_cnn_gather", opsin_ptr, stride, pitch, pw, ph, None, tiles,
                  distance, self.workspace.data_ptr(), _stream())

    def forward(self, tiles: int, tensor_cores: bool = False) -> torch.Tensor:
        """Head outputs [tiles, 64, 28] of the inputs in the workspace (SIMT
        convolutions, or the tensor-core ones the learned analysis runs)."""
        head = torch.empty((tiles, 64, 28), dtype=torch.float32, device="cuda")
        _lib.call("gjxl_b200_cnn_forward", self.params.data_ptr(), tiles,
                  self.workspace.data_ptr(), head.data_ptr(), int(tensor_cores), _stream())
        return head

    def train_step(self, tiles: int, labels: torch.Tensor, targets: torch.Tensor,
                   weights: torch.Tensor, lr: float, weight_decay: float = 1e-4) -> torch.Tensor:
        """Forward, loss, backward and one AdamW step on the workspace's inputs."""
        _lib.call("gjxl_b200_cnn_forward", self.params.data_ptr(), tiles,
                  self.workspace.data_ptr(), None, 0, _stream())
        _lib.call("gjxl_b200_cnn_train_step", self.params.data_ptr(), tiles,
                  self.workspace.data_ptr(), labels.data_ptr(), targets.data_ptr(),
                  weights.data_ptr(), QF_WEIGHT, self.grads.data_ptr(),
                  self.scratch.data_ptr(), self.loss.data_ptr(), _stream())
        self.step += 1
        _lib.call("gjxl_b200_cnn_adamw", self.params.data_ptr(), self.grads.data_ptr(),
                  self.m.data_ptr(), self.v.data_ptr(), self.step, lr, 0.9, 0.999, 1e-8,
                  weight_decay, _stream())
        return self.loss


@dataclass
class Examples:
    inputs: torch.Tensor   # [T, 80, 80, 4] int16 (BF16 bits)
    labels: torch.Tensor   # [T, 64] uint8 strategy codes
    targets: torch.Tensor  # [T, 64] float32 log field corrections
    weights: torch.Tensor  # [T, 64] float32, 0 for block slots outside the image


def tile_targets(cells: np.ndarray, final: np.ndarray, adjusted: np.ndarray, tiles_x: int,
                 tiles_y: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Per tile and block slot (raster within the tile): strategy code, log
    field correction and weight (0 outside the image)."""
    by, bx = cells.shape
    labels = np.zeros((tiles_y * 8, tiles_x * 8), np.uint8)
    targets = np.zeros((tiles_y * 8, tiles_x * 8), np.float32)
    weights = np.zeros((tiles_y * 8, tiles_x * 8), np.float32)
    labels[:by, :bx] = cells >> 1
    targets[:by, :bx] = np.log(final / adjusted)
    weights[:by, :bx] = 1.0
    shape = (tiles_y, 8, tiles_x, 8)
    per_tile = lambda a: a.reshape(shape).transpose(0, 2, 1, 3).reshape(-1, 64)
    return per_tile(labels), per_tile(targets), per_tile(weights)


def examples_from_analysis(session: AnalysisSession, distance: float,
                           network: ProposalNetwork) -> Examples:
    """The training examples of one finished analysis (after analyze_host)."""
    o = session.outputs
    tiles = o.tiles_x * o.tiles_y
    network.gather(o.preprocessed_opsin, o.opsin_stride, o.opsin_plane_pitch, o.padded_width,
                   o.padded_height, tiles, distance)
    inputs = network.inputs(tiles).clone()
    r = session.host_results()
    adjusted = device_array(o.adjusted_quant_field, (o.blocks_y, o.blocks_x), np.float32)
    labels, targets, weights = tile_targets(r["cells"], r["final_quant"],
                                            adjusted.cpu().numpy(), o.tiles_x, o.tiles_y)
    return Examples(inputs, torch.from_numpy(labels).cuda(), torch.from_numpy(targets).cuda(),
                    torch.from_numpy(weights).cuda())


def concat(parts: list[Examples]) -> Examples:
    return Examples(*(torch.cat([getattr(p, f) for p in parts]) for f in
                      ("inputs", "labels", "targets", "weights")))


def build_examples(images: list[np.ndarray], network: ProposalNetwork,
                   distances=DISTANCES, effort: int = 7) -> Examples:
    """Plain analyses of every image at every distance (one session per
    extent, retargeted), and their examples."""
    sessions: dict[tuple[int, int], AnalysisSession] = {}
    parts = []
    for img in images:
        h, w, _ = img.shape
        s = sessions.get((w, h))
        if s is None:
            s = sessions[(w, h)] = AnalysisSession(w, h, effort=effort, tokenize=False)
        for d in distances:
            s.set_butteraugli_target(d)
            s.analyze_host(np.ascontiguousarray(img), _stream())
            torch.cuda.synchronize()
            parts.append(examples_from_analysis(s, d, network))
    for s in sessions.values():
        s.close()
    return concat(parts)


def metrics(network: ProposalNetwork, ex: Examples, batch: int = 512) -> dict:
    """Top-1 / top-3 strategy accuracy (among the searched strategies) and
    the mean absolute error of the field correction, over valid blocks."""
    searched = torch.tensor([0, 6, 7, 4, 10, 11, 5], device="cuda")
    top1 = top3 = mae = count = 0.0
    for start in range(0, ex.inputs.shape[0], batch):
        n = min(batch, ex.inputs.shape[0] - start)
        network.ensure(n)
        network.inputs(n).copy_(ex.inputs[start:start + n])
        head = network.forward(n)
        logits = head[..., :27].index_select(-1, searched)
        order = searched[logits.argsort(-1, descending=True)]
        lab = ex.labels[start:start + n].long()
        w = ex.weights[start:start + n]
        top1 += float(((order[..., 0] == lab).float() * w).sum())
        top3 += float(((order[..., :3] == lab[..., None]).any(-1).float() * w).sum())
        mae += float(((head[..., 27] - ex.targets[start:start + n]).abs() * w).sum())
        count += float(w.sum())
    return {"top1": top1 / count, "top3": top3 / count, "qf_mae": mae / count,
            "blocks": int(count)}


def train(network: ProposalNetwork, ex: Examples, epochs: int = 4, batch: int = 256,
          lr: float = 2e-3, seed: int = 0, log=None) -> list[float]:
    """Minibatch AdamW over shuffled tiles, cosine learning-rate decay."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    total = ex.inputs.shape[0]
    steps = epochs * (total // batch)
    network.ensure(batch)
    losses = []
    step = 0
    for epoch in range(epochs):
        perm = torch.randperm(total, device="cuda", generator=g)
        for k in range(total // batch):
            idx = perm[k * batch:(k + 1) * batch]
            network.inputs(batch).copy_(ex.inputs.index_select(0, idx))
            rate = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(1, steps)))
            loss = network.train_step(batch, ex.labels.index_select(0, idx).contiguous(),
                                      ex.targets.index_select(0, idx).contiguous(),
                                      ex.weights.index_select(0, idx).contiguous(), rate)
            step += 1
            if k % 50 == 0:
                losses.append(float(loss.item()))
        if log is not None:
            log(f"epoch {epoch}: loss {losses[-1]:.4f}")
    return losses


def _generate(spec):
    from .synthetic import generate_srgb8
    w, h, seed = spec
    return generate_srgb8(w, h, seed)


def generate_images(specs, workers: int = 16) -> list[np.ndarray]:
    """Seeded generator images in spawned host processes (start this before
    any CUDA work in the calling process)."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_generate, specs, chunksize=1)


def bd_rate(plain: list[tuple[float, float]], learned: list[tuple[float, float]]) -> float:
    """Bjontegaard delta rate of `learned` against `plain`, each a list of
    (Butteraugli distance, bytes): log-rate as a cubic in distance, the
    mean difference over the common distance range, as a relative rate
    (positive: the learned form spends more bytes at equal distance)."""
    da, ra = np.array([p[0] for p in plain]), np.log([p[1] for p in plain])
    db, rb = np.array([p[0] for p in learned]), np.log([p[1] for p in learned])
    deg = min(3, len(da) - 1)
    pa, pb = np.polyfit(da, ra, deg), np.polyfit(db, rb, deg)
    lo, hi = max(da.min(), db.min()), min(da.max(), db.max())
    ia, ib = np.polyint(pa), np.polyint(pb)
    avg = ((np.polyval(ib, hi) - np.polyval(ib, lo)) -
           (np.polyval(ia, hi) - np.polyval(ia, lo))) / (hi - lo)
    return float(np.exp(avg) - 1.0)


ENCODER_PATH = Path(__file__).resolve().parent.parent / "integration" / "_build" / \
    "libgjxl_b200_encoder.so"


def encode(img: np.ndarray, distance: float, weights: torch.Tensor | None,
           learned_iterations: int = 0, confidence: float = 0.6) -> tuple[int, float, float]:
    """Codestream bytes, final Butteraugli distance (maximum) and its FP64
    3-norm for one encode through the reference's unchanged serializer
    (integration/b200_encoder.cpp); weights None: the plain method."""
    from ctypes import POINTER, c_double, c_float, c_int, c_size_t, c_void_p
    lib = ctypes.CDLL(str(ENCODER_PATH))
    img = np.ascontiguousarray(img)
    h, w, ch = img.shape
    capacity = max(1 << 16, 4 * w * h)
    out = np.empty(capacity, np.uint8)
    size, score, pnorm = c_size_t(0), c_double(0.0), c_double(0.0)
    fn = lib.gjxl_b200_encode_image_learned
    fn.argtypes = [c_void_p, c_size_t, c_size_t, c_size_t, c_int, c_float, c_int, c_int,
                   c_void_p, c_int, c_float, c_void_p, c_size_t, POINTER(c_size_t),
                   POINTER(c_double), POINTER(c_double)]
    rc = fn(img.ctypes.data, w, h, w * ch, ch, distance, 7, 0,
            None if weights is None else weights.data_ptr(), learned_iterations, confidence,
            out.ctypes.data, capacity, ctypes.byref(size), ctypes.byref(score),
            ctypes.byref(pnorm))
    if rc != 0:
        lib.gjxl_b200_integration_last_error.restype = ctypes.c_char_p
        raise RuntimeError(lib.gjxl_b200_integration_last_error().decode())
    return int(size.value), float(score.value), float(pnorm.value)


def analysis_ms(img: np.ndarray, distance: float, weights: torch.Tensor | None,
                learned_iterations: int = 0, reps: int = 10) -> tuple[float, dict]:
    """Device time of one analysis (graph replay, median of `reps`), and the
    share of (tile, family) pairs the learned search kept."""
    h, w, _ = img.shape
    s = AnalysisSession(w, h, butteraugli_target=distance, effort=7,
                        proposal_weights=0 if weights is None else weights.data_ptr(),
                        learned_iterations=learned_iterations)
    d = torch.from_numpy(np.ascontiguousarray(img).reshape(h, -1)).cuda()
    stream = torch.cuda.current_stream()
    for _ in range(3):
        s.analyze(d.data_ptr(), 3 * w, 3, stream.cuda_stream)
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.analyze(d.data_ptr(), 3 * w, 3, stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    info = {}
    if weights is not None:
        o = s.outputs
        masks = device_array(o.tile_family_masks, (o.tiles_y, o.tiles_x), np.uint8).cpu().numpy()
        bits = np.unpackbits(masks[..., None], axis=-1)[..., 1:].sum(-1)
        info = {"families_kept": float(bits.mean() / 7.0),
                "fallback_tiles": float((masks == 0x7F).mean())}
    s.close()
    return float(np.median(times)), info


def evaluate(weights_path: Path, images: list[np.ndarray], learned_iterations: int = 0) -> dict:
    """Learned versus plain on held-out images: BD-rate over DISTANCES and
    the analysis time of each form."""
    net = ProposalNetwork.load(weights_path)
    per_image = []
    for img in images:
        plain = [encode(img, d, None) for d in DISTANCES]
        learned = [encode(img, d, net.params, learned_iterations) for d in DISTANCES]
        ms_plain, _ = analysis_ms(img, 1.0, None)
        ms_learned, info = analysis_ms(img, 1.0, net.params, learned_iterations)
        per_image.append({
            "bd_rate": bd_rate([(s, b) for b, s, _ in plain], [(s, b) for b, s, _ in learned]),
            "bd_rate_pnorm": bd_rate([(q, b) for b, _, q in plain],
                                     [(q, b) for b, _, q in learned]),
            "plain": plain, "learned": learned, "analysis_ms_plain": ms_plain,
            "analysis_ms_learned": ms_learned} | info)
    return {"images": len(images), "learned_iterations": learned_iterations,
            "bd_rate_mean": float(np.mean([p["bd_rate"] for p in per_image])),
            "bd_rate_pnorm_mean": float(np.mean([p["bd_rate_pnorm"] for p in per_image])),
            "speedup_mean": float(np.mean([p["analysis_ms_plain"] / p["analysis_ms_learned"]
                                           for p in per_image])),
            "per_image": per_image}


def main():
    from .synthetic import workload_seed
    parser = argparse.ArgumentParser()
    sub = parser.add_subparsers(dest="command", required=True)
    t = sub.add_parser("train")
    t.add_argument("--images", type=int, default=128)
    t.add_argument("--held-out", type=int, default=16)
    t.add_argument("--size", type=int, default=1024)
    t.add_argument("--epochs", type=int, default=4)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--out", type=Path, required=True)
    e = sub.add_parser("evaluate")
    e.add_argument("--weights", type=Path, default=WEIGHTS_PATH)
    e.add_argument("--images", type=int, default=8)
    e.add_argument("--first", type=int, default=128 + 16)
    e.add_argument("--size", type=int, default=1024)
    e.add_argument("--iterations", type=int, default=0)
    args = parser.parse_args()
    if args.command == "evaluate":
        specs = [(args.size, args.size, workload_seed(5, args.first + i))
                 for i in range(args.images)]
        images = generate_images(specs)
        print(json.dumps(evaluate(args.weights, images, args.iterations)))
        return
    # Configuration 5 seeds: training images 0.., held-out images after them.
    specs = [(args.size, args.size, workload_seed(5, i))
             for i in range(args.images + args.held_out)]
    t0 = time.time()
    images = generate_images(specs)
    t1 = time.time()
    network = ProposalNetwork(seed=1)
    train_ex = build_examples(images[:args.images], network)
    held_ex = build_examples(images[args.images:], network)
    torch.cuda.synchronize()
    t2 = time.time()
    before = metrics(network, held_ex)
    losses = train(network, train_ex, epochs=args.epochs, lr=args.lr, log=print)
    torch.cuda.synchronize()
    t3 = time.time()
    after = metrics(network, held_ex)
    network.save(args.out)
    print(json.dumps({"train_tiles": int(train_ex.inputs.shape[0]),
                      "held_out_tiles": int(held_ex.inputs.shape[0]),
                      "losses": [round(v, 4) for v in losses], "held_out_before": before,
                      "held_out_after": after, "generate_s": round(t1 - t0, 1),
                      "examples_s": round(t2 - t1, 1), "train_s": round(t3 - t2, 1)}))


if __name__ == "__main__":
    main()
