"""CPU pin of oracle/torch_renderer.py, the torch restatement of the
reference's PyTorch per-tile renderer that bench.py's reference arm times:
its image, alpha and the six parameter gradients equal what the reference's
own renderer produced on the same inputs (tests/golden/torch_*.npz, made by
tests/golden/make_golden.py from SimpleTileRenderer._process_tiles_parallel
on the CPU path)."""
import numpy as np
import pytest
import torch

from oracle import torch_renderer as TR
from helpers import golden, split_mapping


@pytest.mark.parametrize("name", ["disk64", "ragged"])
def test_torch_port_matches_reference_renderer(name):
    d = golden(f"torch_{name}")
    H, W, ts = int(d["H"]), int(d["W"]), int(d["ts"])
    offs, idx = split_mapping(d["mapping"])
    leaf = lambda a: torch.tensor(np.ascontiguousarray(a, np.float32), requires_grad=True)
    x, y = leaf(d["means2D"][:, 0]), leaf(d["means2D"][:, 1])
    r, th, v, c = leaf(d["radii"]), leaf(d["rotations"]), leaf(d["opacities"]), leaf(d["colors"])
    img, alpha = TR.render(H, W, ts, x, y, r, th, v, c, torch.from_numpy(d["S"]), torch.from_numpy(d["sel"]),
                           float(d["amax"]), torch.from_numpy(offs), torch.from_numpy(idx))
    assert np.abs(img.detach().numpy() - d["image"]).max() <= 1e-6
    assert np.abs(alpha.detach().numpy() - d["alpha"]).max() <= 1e-6
    ((img * torch.from_numpy(d["wc"])).sum() + (alpha * torch.from_numpy(d["wa"])).sum()).backward()
    for t, key in ((x, "g_x"), (y, "g_y"), (r, "g_r"), (th, "g_theta"), (v, "g_v"), (c, "g_c")):
        ref = d[key]
        err = np.linalg.norm(t.grad.numpy() - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err <= 1e-5, (key, err)
