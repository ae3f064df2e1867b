"""CPU tests of the fit loop's schedules against the reference's own loop.

tests/golden/fit_loop.npz records SimpleTileRenderer._optimize_parameters_whole
(simple_tile_renderer.py:913-1228) run by tests/golden/make_golden.py on the
reference's CPU path with ExponentialLR decay, the adaptive blur schedule and
pruning: per iteration the learning rate of each Adam group at its step and
the blur sigma handed to the renderer, and per prune its iteration, the
opacity logits it saw and the primitives it replaced.  The host statements of
the schedules in diffbmp_b200.fitting (which the device kernels evaluate from
the device step count) must reproduce them; the GPU test
test_gpu_fitting.py::test_loop_decay_blur_prune_step_by_step checks the
device against those statements."""
import json

import numpy as np

from diffbmp_b200 import fitting as F
from helpers import golden


def _cfg(fx):
    return F.FitConfig.from_opt_conf(json.loads(str(fx["conf"])), pool=fx["pool"])


def test_learning_rates_match_reference_loop():
    fx = golden("fit_loop")
    cfg = _cfg(fx)
    N = int(fx["N"])
    want = fx["lrs"]                       # (iterations, 6): x, y, r, v, theta, c
    assert want.shape == (cfg.num_iterations, 6)
    got = np.array([F.lr_schedule(cfg, N, k) for k in range(cfg.num_iterations)])
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    assert cfg.decay_rate == float(fx["decay_rate"]) < 1.0


def test_blur_sigmas_match_reference_loop():
    fx = golden("fit_loop")
    cfg = _cfg(fx)
    got = np.array([F.blur_sigma_at(cfg, k) for k in range(cfg.num_iterations)])
    np.testing.assert_allclose(got, fx["sigmas"], rtol=0, atol=1e-15)
    assert cfg.blur == "adaptive" and got[0] == float(fx["sigma_start"])


def test_prune_schedule_and_selection_match_reference_loop():
    fx = golden("fit_loop")
    cfg = _cfg(fx)
    due = [k for k in range(cfg.num_iterations) if F.prune_due(cfg, k)]
    assert due == fx["prune_its"].tolist()
    start = 0
    for v, n in zip(fx["prune_v"], fx["prune_counts"]):
        want = fx["prune_idx"][start:start + n]
        start += n
        assert np.array_equal(F.prune_selection(cfg, v), want)
    assert start == fx["prune_idx"].size > 0


def test_fixed_blur_and_no_decay_defaults():
    cfg = F.FitConfig.from_opt_conf({"num_iterations": 10, "learning_rate": {"default": 0.1},
                                     "do_gaussian_blur": True, "blur_sigma": 1.5})
    assert cfg.blur == "fixed" and F.blur_sigma_at(cfg, 7) == 1.5
    assert cfg.decay_rate == 1.0 and cfg.prune is None
    assert not any(F.prune_due(cfg, k) for k in range(10))
    lrs = F.lr_schedule(cfg, 100, 5)
    assert lrs[0] == 0.1 * 10.0 and lrs[3] == 0.1 * 1.5 * 10.0
