"""Row N3 host logic: the batch's placement rule (gjxl_b200_batch_schedule)
against a plain restatement of it: order as given or by decreasing pixels
(ties in request order), each request to the lane with the fewest pixels so
far (lowest index on ties). No GPU needed."""

import numpy as np
import pytest

from gjxl_b200 import batch


def restated(pixels, lanes, largest_first):
    order = sorted(range(len(pixels)), key=lambda i: -pixels[i]) if largest_first \
        else list(range(len(pixels)))
    load = [0] * lanes
    lane_of = [0] * len(pixels)
    for i in order:
        lane = min(range(lanes), key=lambda l: (load[l], l))
        lane_of[i] = lane
        load[lane] += pixels[i]
    return lane_of, order


@pytest.mark.parametrize("lanes", [1, 2, 3, 8, 16])
@pytest.mark.parametrize("largest_first", [False, True])
def test_schedule_matches_restatement(lanes, largest_first):
    rng = np.random.default_rng(lanes * 2 + largest_first)
    sides = np.exp(rng.uniform(np.log(256), np.log(4096), (64, 2))).astype(np.int64)
    pixels = list(sides[:, 0] * sides[:, 1])
    pixels[5] = pixels[9]  # a tie
    lane_of, order = batch.schedule(pixels, lanes, largest_first)
    want_lane, want_order = restated(pixels, lanes, largest_first)
    assert list(order) == want_order
    assert list(lane_of) == want_lane


def test_schedule_balances_load():
    pixels = [4096 * 4096] + [256 * 256] * 63
    lane_of, _ = batch.schedule(pixels, 4, True)
    assert lane_of[0] == 0 and all(l != 0 for l in lane_of[1:])


def test_schedule_rejects_bad_lanes():
    from gjxl_b200._lib import GjxlB200Error
    with pytest.raises(GjxlB200Error):
        batch.schedule([1, 2, 3], 0, False)
    with pytest.raises(GjxlB200Error):
        batch.schedule([1, 2, 3], 17, False)
