"""Host-side scene builders and post-processing: marker rings, seeded
non-overlapping cylinder sets, the Strouhal estimator."""
import math

import numpy as np
import pytest

from ippi_lbm import scenes
from ippi_lbm.learned_tau import strouhal
from ippi_lbm.validation import config3_scene, seeded_cylinders


def test_cylinder_markers_ring():
    xy, ds = scenes.cylinder_markers(100.0, 50.0, 20)
    assert len(ds) == 63 and xy.shape == (63, 2)  # ceil(pi D)
    r = np.hypot(xy[:, 0] - 100.0, xy[:, 1] - 50.0)
    np.testing.assert_allclose(r, 10.0, rtol=1e-14)
    assert ds.sum() == pytest.approx(math.pi * 20)
    # marker 0 at the top, as Mesh::InitialIBParticle (x = cx + r sin, y = cy + r cos)
    assert xy[0] == pytest.approx([100.0, 60.0])


@pytest.mark.parametrize("period", [1600.0, 1234.5, 5333.3])
def test_strouhal_resolves_below_one_bin(period):
    t = np.arange(20000)
    cl = np.sin(2 * np.pi * t / period + 0.3) + 0.2 * np.sin(4 * np.pi * t / period)
    # a few periods in the record (3.75 for the longest): 1e-3; one bin is 6.7 %
    assert strouhal(cl, 20, 0.05) == pytest.approx(20 / (0.05 * period), rel=1e-3)


def test_seeded_cylinders_keep_their_gap():
    c = seeded_cylinders(16384, 4096, 48, 64, 96, seed=0)
    d = np.hypot(c[:, None, 0] - c[None, :, 0], c[:, None, 1] - c[None, :, 1])
    assert d[np.triu_indices(64, 1)].min() >= 48 + 96
    assert c[:, 0].min() >= 3 * 48 and c[:, 1].min() >= 2 * 48 and c[:, 1].max() <= 4096 - 2 * 48
    np.testing.assert_array_equal(c, seeded_cylinders(16384, 4096, 48, 64, 96, seed=0))


def test_config3_scene_bodies():
    sc = config3_scene(2048, 512, d=48, n=4)
    assert sc["bodies"].max() == 3 and len(sc["bodies"]) == len(sc["ds"]) == 4 * 151


def test_bench_modes_resolve_their_drivers():
    """Every driver function the bench's learned and adjoint modes call is
    present in the package (import-level check; the runs need a GPU)."""
    import inspect

    from ippi_lbm import learned_tau as lt
    from ippi_lbm.autograd import NetworkRollout, Rollout

    assert callable(NetworkRollout.apply) and inspect.isclass(Rollout)
    sig = inspect.signature(lt.experiment)
    for k in ("fine_steps", "avg_steps", "device", "finetune_iters"):
        assert k in sig.parameters, k
    assert "iters" in inspect.signature(lt.train_through_solver).parameters


def test_output_scale_calibration_finds_the_closest_drag(monkeypatch):
    """calibrate_scale on a synthetic drag curve Cd(scale) (a bump in
    log(scale), the shape the coarse channel shows): the target inside the
    curve's range is met closely, one above its peak gets the peak."""
    from ippi_lbm import learned_tau as lt

    def fake_run(sc, steps, avg_from, net=None, device=0):
        return dict(cd=0.96 + 0.47 * math.exp(-((math.log(net.out_scale) - math.log(300)) / 2.5) ** 2))

    monkeypatch.setattr(lt, "run_cylinder", fake_run)
    net = lt.TauNet(np.zeros(1313), np.zeros(6), np.ones(6), np.zeros(6), np.ones(6), 2.0)
    best, hist = lt.calibrate_scale(net, None, 1.63, 10, 1)
    assert len(hist) <= 6 + 6 and best.w is not None
    assert abs(best.out_scale - 300) < 30  # the peak, 1.43
    best, hist = lt.calibrate_scale(net, None, 1.2, 10, 1)
    assert min(abs(c - 1.2) for _, c in hist) < 0.002
    assert fake_run(None, 0, 0, best)["cd"] == pytest.approx(1.2, abs=0.002)
