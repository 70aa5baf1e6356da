"""Bench bookkeeping that needs no GPU: the algorithmic FP64 work behind the
roofline figure, and the crops of the timed CPU baseline."""

import bench


def anchors_in_tile(tw: int, th: int, cw: int, ch: int, step: int) -> int:
    """Anchors of one transform family in a tile of tw x th blocks: positions
    on the family's step grid (within the 8x8 tile) whose footprint fits."""
    xs = [x for x in range(0, 8, step) if x + cw <= min(8, tw)]
    ys = [y for y in range(0, 8, step) if y + ch <= min(8, th)]
    return len(xs) * len(ys)


def test_candidate_cost_operations_match_the_candidate_set():
    bx, by = bench.WIDTH // 8, bench.HEIGHT // 8
    total = 0
    for w, h, cw, ch, step in bench.FAMILIES:
        anchors = sum(anchors_in_tile(min(8, bx - tx), min(8, by - ty), cw, ch, step)
                      for ty in range(0, by, 8) for tx in range(0, bx, 8))
        # Forward and inverse separable DCT of 3 channels: (W + H) multiply-adds
        # per coefficient, each multiply and add counted as one operation.
        total += anchors * 3 * 2 * (w * h) * (w + h) * 2
    assert bench.candidate_cost_fp64_ops(bx, by) == total
    # The figure quoted with the roofline for the 4032x3024 workload.
    assert total == 70_894_559_232


def test_reference_crops_tile_the_workload_image():
    crops = bench.reference_crops(16)
    assert len(crops) == 16
    for x, y in crops:
        assert 0 <= x <= bench.WIDTH - bench.CROP_W
        assert 0 <= y <= bench.HEIGHT - bench.CROP_H
    # Distinct crops while the image holds enough of them.
    cols, rows = bench.WIDTH // bench.CROP_W, bench.HEIGHT // bench.CROP_H
    assert len(set(bench.reference_crops(cols * rows))) == cols * rows
