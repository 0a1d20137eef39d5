"""Module-level validation drivers, restated from the reference's
Validation/Hydrodynamics/LocalInertial_CA_Phase1/run_local_inertial_ca_hydrodynamics_validation.m
(plane :44-135, V-tilt :136-218, Ritter :219-297; the LI step at :395-415, fixed dt, rain added
to h before each step, outlet Manning sink with outlet_type 1).

`step_fn(h, dt_s) -> (h_new, q_out_m3_s)` abstracts the routing step so the same driver runs
the literal FP64 restatement, the kernel-form restatement (float/double) or the GPU library.
"""
from __future__ import annotations

import math

import numpy as np

from oracle import literal as L


# ---------------------------------------------------------------- step implementations
class LiteralStep:
    def __init__(self, z, n, dx, rows, cols, slope):
        self.z, self.n, self.dx = z, n, dx
        self.rows, self.cols, self.slope = rows, cols, slope
        self.outflow = np.zeros((3,) + z.shape)

    def __call__(self, h, dt_s):
        dx = self.dx
        out = L.local_inertial_model_d4(self.z, h * 1000, self.n, self.n * self.n, dx * dx, dt_s / 60, dx,
                                        self.rows, self.cols, 1, self.slope, self.outflow)
        self.outflow = out.outflow
        return np.fmax(out.d_t / 1000, 0), out.outlet_flow.sum() / 1000 / 3600 * dx * dx


class SurfaceStep:
    """Kernel-form oracle or the GPU library through the unfused hp2d_li_step."""

    def __init__(self, sf, z, n, dx, rows, cols, slope):
        self.sf = sf
        self.dx = dx
        sf.upload_static(z, n, rows, cols)
        sf.set_state(np.zeros(z.shape))

    def __call__(self, h, dt_s):
        sf = self.sf
        q = (sf.download_native("qx").astype(np.float64) * 3.6e6 / self.dx,
             sf.download_native("qy").astype(np.float64) * 3.6e6 / self.dx)
        sf.set_state(h * 1000, np.stack(q))
        sf.li_step(dt_s / 60)
        hn = np.fmax(sf.download_native("h").astype(np.float64), 0)
        qo = sf.download_native("qo").astype(np.float64).sum() * self.dx * self.dx
        return hn, qo


# ---------------------------------------------------------------- cases
def plane_case():
    dx, nx, ny, S, nman = 20.0, 50, 5, 0.005, 0.035
    x = (np.arange(1, nx + 1) - 0.5) * dx
    z = np.tile(x.max() * S - x * S, (ny, 1))
    return dict(z=z, n=np.full((ny, nx), nman), dx=dx, rows=np.arange(ny), cols=np.full(ny, nx - 1), slope=S,
                rain=40.0, duration=2 * 3600.0, dt=1.0, S=S, nman=nman)


def vtilt_case():
    dx, nx, ny = 20.0, 41, 31
    cc, rr = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1))
    center = math.ceil(nx / 2)
    z = 0.02 * np.abs(cc - center) * dx + 0.004 * (ny - rr) * dx
    cols = np.arange(center - 2, center + 1)          # center_col-1:center_col+1, 0-based
    return dict(z=z, n=np.full((ny, nx), 0.04), dx=dx, rows=np.full(cols.size, ny - 1), cols=cols, slope=0.004,
                rain=30.0, duration=90 * 60.0, dt=1.0, center=center)


def ritter_case():
    dx, nx, ny, dam, h0 = 2.0, 251, 5, 180.0, 1.0
    x = (np.arange(1, nx + 1) - 0.5) * dx
    return dict(z=np.zeros((ny, nx)), n=np.zeros((ny, nx)), dx=dx, rows=np.zeros(0, int), cols=np.zeros(0, int),
                slope=0.001, x=x, dam=dam, h0=h0, h_init=np.tile((x < dam).astype(float) * h0, (ny, 1)))


# ---------------------------------------------------------------- drivers
def run_plane(step):
    c = plane_case()
    ny, nx = c["z"].shape
    rain = c["rain"] / 1000 / 3600
    Lm, W = nx * c["dx"], ny * c["dx"]
    a = (1 / c["nman"]) * math.sqrt(c["S"])
    tc = (Lm / (a * rain ** (2 / 3))) ** (3 / 5)

    def kq(t):  # kinematic_plane_q, run_local_inertial_ca_hydrodynamics_validation.m:523-538
        return W * (a * (rain * t) ** (5 / 3) if t < tc else rain * Lm)

    h = np.zeros((ny, nx))
    qm, qa, mass, cum = [], [], [], 0.0
    for it in range(1, int(round(c["duration"] / c["dt"])) + 1):
        h = h + rain * c["dt"]
        h, qo = step(h, c["dt"])
        cum += qo * c["dt"]
        if it % 60 == 0:
            t = it * c["dt"]
            qm.append(qo)
            qa.append(kq(t))
            rv = rain * t * nx * ny * c["dx"] ** 2
            mass.append(100 * (h.sum() * c["dx"] ** 2 + cum - rv) / rv)
    qm, qa = np.array(qm), np.array(qa)
    nse = 1 - np.sum((qm - qa) ** 2) / np.sum((qa - qa.mean()) ** 2)
    return dict(nse=nse, rel_l2=np.linalg.norm(qm - qa) / np.linalg.norm(qa), mass_pct=float(np.max(np.abs(mass))))


def run_vtilt(step):
    c = vtilt_case()
    ny, nx = c["z"].shape
    rain = c["rain"] / 1000 / 3600
    h = np.zeros((ny, nx))
    sym, mass, cum = [], [], 0.0
    k = c["center"]
    for it in range(1, int(round(c["duration"] / c["dt"])) + 1):
        h = h + rain * c["dt"]
        h, qo = step(h, c["dt"])
        cum += qo * c["dt"]
        if it % 60 == 0:
            left = h[:, :k - 1]
            right = np.fliplr(h[:, k:])
            sym.append(math.sqrt(np.mean((left - right) ** 2)))
            rv = rain * it * c["dt"] * nx * ny * c["dx"] ** 2
            mass.append(100 * (h.sum() * c["dx"] ** 2 + cum - rv) / rv)
    return dict(symmetry_rmse=max(sym), mass_pct=float(np.max(np.abs(mass))), channel_depth=float(h[:, k - 1].mean()))


def run_ritter(step):
    c = ritter_case()
    g = 9.81
    x = c["x"]
    h = c["h_init"].copy()
    rm, rl = [], []
    for it in range(1, 401):
        h, _ = step(h, 0.05)
        if it in (100, 200, 300, 400):
            t = it * 0.05
            prof = h.mean(0)
            c0 = math.sqrt(g * c["h0"])
            xi = x - c["dam"]
            ref = np.zeros_like(x)
            ref[xi <= -c0 * t] = c["h0"]
            fan = (xi > -c0 * t) & (xi < 2 * c0 * t)
            ref[fan] = (2 * c0 - xi[fan] / t) ** 2 / (9 * g)     # ritter_depth, :540-548
            act = (x >= c["dam"] - c0 * t - 5 * c["dx"]) & (x <= c["dam"] + 2 * c0 * t + 5 * c["dx"])
            err = prof - ref
            rm.append(math.sqrt(np.mean(err[act] ** 2)))
            rl.append(np.linalg.norm(err[act]) / np.linalg.norm(ref[act]))
    return dict(rmse=max(rm), rel_l2=max(rl))
