"""Row N4: what the trained proposal network (the committed weights) gains
over the plain method, on held-out images it never saw (1024x1024, seeds of
the network's configuration after its training and evaluation images):
the learned analysis (proposed families only in confident tiles, one field
update from the predicted field) is faster than the plain analysis (two
field updates, full search), searches fewer candidate families, and its
codestreams through the reference's serializer cost about the same bytes at
equal Butteraugli distance (BD-rate over distances 0.5, 1, 2, 3)."""

import pytest

from gjxl_b200 import learned
from gjxl_b200.synthetic import generate_srgb8, workload_seed

pytestmark = pytest.mark.gpu


def test_learned_form_gains_over_plain(cuda):
    held = [generate_srgb8(1024, 1024, workload_seed(5, 2000 + i)) for i in range(2)]
    ev = learned.evaluate(learned.WEIGHTS_PATH, held, learned_iterations=1)
    for p in ev["per_image"]:
        assert p["families_kept"] < 0.95, p
        assert p["analysis_ms_learned"] < 0.95 * p["analysis_ms_plain"], p
    # The target is at most 0.5% over a larger held-out set; two images
    # bound it loosely.
    assert ev["bd_rate_pnorm_mean"] <= 0.02, ev["bd_rate_pnorm_mean"]
    assert ev["bd_rate_mean"] <= 0.05, ev["bd_rate_mean"]


def test_bd_rate_restatement():
    curve = [(0.5, 1000.0), (1.0, 600.0), (2.0, 350.0), (3.0, 250.0)]
    assert abs(learned.bd_rate(curve, curve)) < 1e-12
    assert abs(learned.bd_rate(curve, [(d, b * 1.03) for d, b in curve]) - 0.03) < 1e-9
