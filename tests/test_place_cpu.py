"""Placement of boxes and jobs on the GPUs of a node (mdpd_place: host only, no GPU).

Each item lands on exactly one device or on none (-1, MDPD_ERR_BUDGET); no device's bytes exceed
its budget; the work (particles, or particles times steps) is balanced by longest-processing-time
first; the same inputs always give the same placement, so ranks need not exchange it."""
import numpy as np
import pytest

import mdpd
import bench


def specs(seed=1, nbox=256):
    return bench.specs_of(bench.batched_boxes(seed=seed, nbox=nbox))


def test_every_box_placed_once_and_balanced():
    sp = specs(nbox=512)
    for ndev in (2, 4, 8):
        dev, work = mdpd.place(sp, ndev, int(150e9))
        assert dev.min() >= 0 and dev.max() < ndev
        n = np.array([s.n for s in sp], float)
        per = np.bincount(dev, weights=n, minlength=ndev)
        assert np.allclose(per, work)
        assert per.max() / per.min() < 1.01, per  # 512 uneven boxes: LPT balances within 1%
        assert per.sum() == n.sum()


def test_jobs_weighted_by_steps_and_budget_respected():
    sp = specs(seed=2, nbox=64)
    rng = np.random.default_rng(3)
    steps = rng.integers(2000, 20001, len(sp))
    foot = np.array([mdpd.box_bytes(s) for s in sp])
    budget = int(foot.sum() / 4 * 1.1)  # 4 devices with 10% headroom
    dev, work = mdpd.place(sp, 4, budget, steps=steps)
    for d in range(4):
        assert foot[dev == d].sum() <= budget
    w = np.array([s.n for s in sp], float) * steps
    assert np.allclose(np.bincount(dev, weights=w, minlength=4), work)
    # unequal budgets: a device with no room takes nothing
    dev2, _ = mdpd.place(sp, 3, [int(foot.sum()), 0, int(foot.sum())], steps=steps)
    assert not np.any(dev2 == 1)


def test_box_that_fits_nowhere_is_reported():
    sp = specs(nbox=8)
    foot = np.array([mdpd.box_bytes(s) for s in sp])
    big = int(np.argmax(foot))
    with pytest.raises(mdpd.MdpdError) as e:
        mdpd.place(sp, 2, int(foot[big] - 1))
    assert e.value.code == mdpd.ERR_BUDGET


def test_placement_is_deterministic():
    sp = specs(nbox=300)
    a, _ = mdpd.place(sp, 4, int(150e9))
    b, _ = mdpd.place(sp, 4, int(150e9))
    assert np.array_equal(a, b)
