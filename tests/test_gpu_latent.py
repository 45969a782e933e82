"""fb_probit_latent_device, fpbart's latent redraw (src/bart_kernel.cpp:280-292, 543-547) on its own: bit-exact against
the oracle's restatement of the sampler's draw (same counters: chain seed, row, sweep), the truncation on the right
side of -offset for each outcome, the initial draw (sweep -1, fit 0), ragged sizes and tail cases."""
import numpy as np
import pytest

import fastbart_b200 as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,sweep,offset,scale", [(1, 0, 0.0, 1.0), (1000, 17, 0.3, 1.0), (65537, 999, -0.7, 3.0),
                                                  (4099, -1, 0.25, 0.0), (2000, 5, 4.0, 0.5)])
def test_latent_redraw_bit_exact(orc, n, sweep, offset, scale):
    import torch
    rng = np.random.default_rng(n + sweep)
    fit = rng.normal(0.0, scale, n)   # scale 3: tails far beyond the truncation point
    ybin = (rng.random(n) < 0.5).astype(np.int32)
    seed = 0x9E3779B97F4A7C15 + n
    fd = torch.tensor(fit, device="cuda")
    yd = torch.tensor(ybin, device="cuda")
    zd = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    cap = torch.zeros(1, dtype=torch.int32, device="cuda")
    F.probit_latent_device(fd.data_ptr(), yd.data_ptr(), n, offset, seed, sweep, zd.data_ptr(), cap.data_ptr())
    torch.cuda.synchronize()
    z = zd.cpu().numpy()
    ref, caps = orc.probit_latent(seed, sweep, offset, fit, ybin)
    assert np.array_equal(z, ref)
    assert int(cap.item()) == caps
    assert np.all(z[ybin == 1] > -offset) and np.all(z[ybin == 0] < -offset)
