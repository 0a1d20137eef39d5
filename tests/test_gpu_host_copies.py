"""Host copies at the C ABI: pageable caller arrays of 32 MiB and more are staged through the
context's page-locked chunks by several host threads; page-locked arrays go in one copy.  Both
routes must carry the same bits, including a last chunk shorter than the others."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned(shape):
    import torch
    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


@pytest.mark.parametrize("shape", [(2048, 2048), (2100, 2051)])   # 32 MiB exactly; ragged chunks
def test_pageable_and_page_locked_copies_agree(shape, hp2d_lib):
    from hydropol2d_b200 import SurfaceFlow
    rng = np.random.default_rng(shape[0])
    z = rng.uniform(0.0, 5.0, shape)
    rough = np.full(shape, 0.03)
    d = rng.uniform(0.0, 500.0, shape)
    rows = np.arange(shape[0], dtype=np.int32)
    cols = np.full(shape[0], shape[1] - 1, dtype=np.int32)
    out = {}
    for route in ("pageable", "page_locked"):
        g = SurfaceFlow(*shape, 2.0, "fp64")
        if route == "page_locked":
            zp, dp = _pinned(shape), _pinned(shape)
            zp[...] = z
            dp[...] = d
            g.upload_static(zp, rough, rows, cols)
            g.set_state(dp)
        else:
            g.upload_static(z, rough, rows, cols)
            g.set_state(d)
        g.fused_steps(3)
        depth = _pinned(shape) if route == "page_locked" else np.empty(shape)
        g.download_into("depth", depth)
        out[route] = (np.array(depth), g.download_native("h"), g.download("dmax"))
        g.close()
    for a, b in zip(out["pageable"], out["page_locked"]):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert np.all(np.isfinite(out["pageable"][0]))
