"""Named synthetic workloads for profiling and timing (each prints one line).

    python -m hydropol2d_b200.workloads wet [--steps N]        fully wet 2048 x 2048 grid
    python -m hydropol2d_b200.workloads dambreak [--ny R]      the bench's dam-break on R x 8192 cells
    python -m hydropol2d_b200.workloads unet [--batch B]        U-Net forward + training step
    python -m hydropol2d_b200.workloads ensemble [--members M]  batched ensemble, a few launches

``wet``: the V-tilted catchment geometry on 2048 x 2048 cells (dx 10 m) plus a 0.5 m random
field, 5 cm of water everywhere and 60 mm/h of rain, so every cell takes the full local-inertial
path of the fused step (no dry-row shortcuts).  ``unet``: the screening network on a batch of
256 x 256 tiles.  ``ensemble``: the 256-member configuration's first launches.
"""
from __future__ import annotations

import argparse

import numpy as np


def wet(steps: int) -> str:
    from . import SurfaceFlow, synthetic as S
    z, ch = S.vtilt_domain(2048, 2048, 10.0, 0.005, 0.002)
    z = z + 0.5 * S.gaussian_random_field(2048, 2048, -3.0, 5)
    p = dict(routing_time=600.0, alfa_min=0.7, alfa_max=0.7, outlet_type=1, slope_outlet=0.002,
             min_time_step=0.01, max_time_step=10.0)
    case = S.Case("wet2048", z, np.full(z.shape, 0.03), 10.0, np.zeros(ch.size, dtype=np.int32),
                  ch.astype(np.int32), p, np.full(z.shape, 50.0),
                  rain_uniform=(np.array([0.0]), np.array([60.0])))
    g = SurfaceFlow(2048, 2048, 10.0, "fp32", **p)
    case.apply(g)
    g.fused_steps(steps)
    ms = g.fused_steps_timed(200)
    g.close()
    return "wet 2048^2: %.4f ms/step, %.1f GCUPS" % (ms / 200, 2048 * 2048 * 200 / ms / 1e6)


def dambreak(ny: int, steps: int) -> str:
    """The dam-break of the benchmark on ny x 8192 cells (the bench's rows when ny = 4096)."""
    from . import SurfaceFlow, synthetic as S
    case = S.dambreak_case(ny, 8192, 5.0, seed=11)
    g = SurfaceFlow(ny, 8192, 5.0, "fp32", **case.params)
    case.apply(g)
    g.fused_steps(steps)
    ms = g.fused_steps_timed(200)
    g.close()
    return "dambreak %dx8192: %.4f ms/step, %.1f GCUPS" % (ny, ms / 200, ny * 8192 * 200 / ms / 1e6)


def unet(batch: int) -> str:
    import torch
    from . import nn
    from .surrogate import UNet, forward_flops
    net = UNet(seed=0)
    x = torch.randn(batch, 256, 256, 4, device="cuda").to(torch.bfloat16)
    for _ in range(3):
        net.predict(x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        net.predict(x)
    e1.record()
    torch.cuda.synchronize()
    ms_f = e0.elapsed_time(e1) / 10
    f = forward_flops(256, 256) * batch
    t = torch.randn(batch * 256 * 256, 2, device="cuda")
    w = torch.ones_like(t)
    for _ in range(3):
        net.train_step(x, t, w, 1e-4)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        net.train_step(x, t, w, 1e-4)
    e1.record()
    torch.cuda.synchronize()
    ms_t = e0.elapsed_time(e1) / 5
    nn.check()
    return ("unet B=%d 256^2: forward %.3f ms (%.1f TFLOP/s), training step %.3f ms (%.1f TFLOP/s, 3x forward)"
            % (batch, ms_f, f / ms_f / 1e9, ms_t, 3 * f / ms_t / 1e9))


def ensemble(members: int, launches: int) -> str:
    from . import SurfaceFlow, synthetic as S
    from .ensemble import Ensemble
    ens = Ensemble()
    for i in range(members):
        c = S.ensemble_member(i)
        g = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
        c.apply(g)
        ens.add(g)
    ens.set_tuning(64)
    ens.steps(4)
    _, ms = ens.steps_timed(launches)
    cells = ens.cells()
    ens.close()
    return "ensemble %d members: %.4f ms/launch, %.1f GCUPS" % (members, ms / launches, cells * launches / ms / 1e6)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["wet", "dambreak", "unet", "ensemble"])
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--launches", type=int, default=64)
    a = ap.parse_args()
    if a.workload == "wet":
        print(wet(a.steps), flush=True)
    elif a.workload == "dambreak":
        print(dambreak(a.ny, a.steps), flush=True)
    elif a.workload == "unet":
        print(unet(a.batch), flush=True)
    else:
        print(ensemble(a.members, a.launches), flush=True)


if __name__ == "__main__":
    main()
