"""CPU tests of the serving loop's host-side sizing: the tile-list bound a job
is admitted and set up with (serving.list_capacity_bound), checked against
the oracle's binning of the same jobs in both content modes, and the
resident-memory estimate built on it.  A bound below the true length would
make every step of the job overflow and replay; the server sizes lists and
admits jobs by HBM budget from these numbers without reading the device."""
import numpy as np
import pytest

from diffbmp_b200 import serving, workloads as wl
from oracle import oracle as O


def _jobs(seed, n, sizes=(96, 160, 256, 512), n_range=(16, 900)):
    rng = np.random.default_rng(seed)
    atlas = np.stack([wl.random_shape(rng, 64) for _ in range(4)])
    return atlas, [wl.make_job(rng, atlas, sizes, n_range) for _ in range(n)]


@pytest.mark.parametrize("mode", [O.BIN_CONTENT, O.BIN_CONTENT_REF])
def test_list_capacity_bound_covers_oracle_lists(mode):
    atlas, jobs = _jobs(5, 10)
    tb = O.template_bboxes(atlas)
    P, Ht, Wt = atlas.shape
    for k, s in enumerate(jobs):
        if k == 1:                      # non-finite geometry and radii past the canvas
            s.rotations[:3] = np.nan
            s.means2D[3] = np.inf
            s.radii[4:8] = 4.0 * max(s.H, s.W)
        if k == 2:                      # degenerate radii
            s.radii[:] = 1e-4
        offs, _ = O.bin_tiles(s.H, s.W, 32, s.means2D, s.radii, s.rotations, s.sel, tb, Ht, Wt, mode)
        bound = serving.list_capacity_bound(s)
        assert bound >= int(offs[-1]), (k, bound, int(offs[-1]))


def test_estimate_bytes_counts_the_list_bound():
    _, jobs = _jobs(6, 4)
    for s in jobs:
        est = serving.estimate_bytes(s)
        # target and background (f32 RGB), per-pixel state, lists at the bound
        assert est >= 2 * s.H * s.W * 12 + s.H * s.W * 8 + 4 * serving.list_capacity_bound(s)
