"""Surrogate screening of ensemble members (no counterpart in the reference).

Pipeline: the batched solver (``Ensemble``) produces peak-depth and arrival-time maps of
training members; three independently initialised U-Nets (``surrogate.UNet``) learn them;
for new members the networks predict the peak depth, and members on which the networks
disagree by more than a threshold go back to the solver.

Inputs per cell (4 channels, FP32-normalised, then BF16): standardised elevation, Manning
n / 0.05, event rain depth (rate x duration) / 100 mm, initial depth / 10 m.  Targets:
log1p(peak depth / 1 cm) and arrival time / routing_time (cells never reached: 1.5 with a
small weight).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from . import nn
from .ensemble import Ensemble
from .surface import SurfaceFlow
from .surrogate import UNet

DEPTH_SCALE_M = 0.01


def member_inputs(case) -> np.ndarray:
    z = np.asarray(case.z, dtype=np.float64)
    zn = (z - np.nanmean(z)) / (np.nanstd(z) + 1e-6)
    n = np.asarray(case.roughness, dtype=np.float64) / 0.05
    rain = 0.0
    if case.meta.get("kind") == "rain":
        rain = case.meta["rate"] * case.meta["duration"] / 60.0 / 100.0
    h0 = np.asarray(case.d0, dtype=np.float64) / 1000.0 / 10.0
    x = np.stack([zn, n, np.full(z.shape, rain), h0], axis=-1)
    return np.nan_to_num(x).astype(np.float32)


def member_targets(dmax_mm: np.ndarray, arrival_min: np.ndarray, routing_min: float):
    d = np.maximum(np.nan_to_num(dmax_mm, nan=0.0, neginf=0.0), 0.0) / 1000.0
    t0 = np.log1p(d / DEPTH_SCALE_M)
    fin = np.isfinite(arrival_min)
    t1 = np.where(fin, np.minimum(arrival_min / routing_min, 1.5), 1.5)
    tgt = np.stack([t0, t1], axis=-1).astype(np.float32)
    w = np.stack([np.ones_like(t0), np.where(fin, 1.0, 0.1)], axis=-1).astype(np.float32)
    return tgt, w


MAX_DEPTH_M = 100.0


def decode_depth_m(pred0) -> np.ndarray:
    """Peak depth [m] from the network's first output (clipped to [0, 100 m])."""
    t = np.clip(np.asarray(pred0, dtype=np.float64), 0.0, np.log1p(MAX_DEPTH_M / DEPTH_SCALE_M))
    return np.expm1(t) * DEPTH_SCALE_M


def peak_m(dmax_mm) -> np.ndarray:
    return np.maximum(np.nan_to_num(np.asarray(dmax_mm, dtype=np.float64), nan=0.0, neginf=0.0), 0.0) / 1000.0


@dataclass
class SolveResult:
    dmax_mm: list
    arrival_min: list
    seconds: float       # device time of the runs
    cell_updates: int


def solve_members(cases, rows_per_warp: int = 16, precision: str = "fp32") -> SolveResult:
    """Runs every member to its routing_time: FP32 members share one batched ensemble,
    FP64 members (the reference's precision) run one after another."""
    t_dev = 0.0
    cu = 0
    if precision == "fp32":
        ens = Ensemble()
        for c in cases:
            g = SurfaceFlow(*c.shape, c.resolution, "fp32", **c.params)
            c.apply(g)
            ens.add(g)
        ens.set_tuning(rows_per_warp)
        active = len(cases)
        while active:
            active, ms = ens.steps_timed(256)
            t_dev += ms / 1e3
        cu = ens.cell_updates()
        out = SolveResult([g.download("dmax") for g in ens.members], [g.download("arrival") for g in ens.members],
                          t_dev, cu)
        ens.close()
        return out
    dm, ar = [], []
    for c in cases:
        g = SurfaceFlow(*c.shape, c.resolution, precision, **c.params)
        c.apply(g)
        t0 = time.perf_counter()
        g.run()
        t_dev += time.perf_counter() - t0
        cu += c.z.size * (g.diag()["k"] - 1)
        dm.append(g.download("dmax"))
        ar.append(g.download("arrival"))
        g.close()
    return SolveResult(dm, ar, t_dev, cu)


class Screener:
    """``n_models`` U-Nets trained on the same data from different initialisations and
    batch orders."""

    def __init__(self, n_models: int = 3, seed: int = 0, base: int = 32, device="cuda"):
        self.models = [UNet(seed=seed + 101 * k, base=base, device=device) for k in range(n_models)]
        self.device = device

    @staticmethod
    def _bf16(x: np.ndarray, device) -> torch.Tensor:
        return torch.from_numpy(np.ascontiguousarray(x)).to(device).to(torch.bfloat16)

    def fit(self, X: np.ndarray, T: np.ndarray, Wt: np.ndarray, epochs: int = 10, batch: int = 16,
            lr: float = 1e-3, seed: int = 0, warmup: int = 200, log=None) -> list:
        """X [N, H, W, 4], T / Wt [N, H, W, 2]; Adam with a linear warm-up over ``warmup``
        steps and cosine decay; returns the mean loss of each epoch per model."""
        N = X.shape[0]
        Xd = self._bf16(X, self.device)
        Td = torch.from_numpy(T.reshape(N, -1, T.shape[-1])).to(self.device)
        Wd = torch.from_numpy(Wt.reshape(N, -1, Wt.shape[-1])).to(self.device)
        rng = np.random.default_rng(seed)
        hist = []
        nb = max(1, N // batch)
        steps_total = epochs * nb
        step = 0
        for ep in range(epochs):
            order = [rng.permutation(N) for _ in self.models]
            losses = [torch.zeros(1, device=self.device) for _ in self.models]
            for b in range(nb):
                lr_t = lr * min(1.0, (step + 1) / warmup) * 0.5 * (1 + np.cos(np.pi * step / steps_total))
                for k, m in enumerate(self.models):
                    idx = torch.from_numpy(order[k][b * batch:(b + 1) * batch]).to(self.device)
                    x = Xd.index_select(0, idx)
                    t = Td.index_select(0, idx).reshape(-1, T.shape[-1])
                    w = Wd.index_select(0, idx).reshape(-1, Wt.shape[-1])
                    losses[k] += m.train_step(x, t, w, lr_t)
                step += 1
            ep_loss = np.array([float(v.item()) / nb for v in losses])
            hist.append(ep_loss)
            if log:
                log(f"epoch {ep}: loss {np.round(ep_loss, 5).tolist()}")
        nn.check()
        return hist

    def predict_timed(self, X: np.ndarray, batch: int = 32, threshold_m: float | None = None,
                      quantile: float = 0.99):
        """Device time [s] of the inference of all members by all models (inputs already on
        the device, outputs left there until the timing ends) and the predictions
        [n_models, N, H, W, 2].  With ``threshold_m`` the disagreement screen runs on the
        device inside the timed region too (``screen_device``) and its (mean peak depth,
        disagreement, rerun mask) follow as a third item."""
        N, H, W, _ = X.shape
        Xd = self._bf16(X, self.device)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        outs = []
        screened = None
        e0.record()
        for s in range(0, N, batch):
            x = Xd[s:s + batch]
            outs.append([m.predict(x) for m in self.models])
        if threshold_m is not None:
            depth0 = torch.stack([torch.cat([o[k].reshape(-1, H * W, o[k].shape[-1])[..., 0] for o in outs])
                                  for k in range(len(self.models))])
            screened = self.screen_device(depth0, threshold_m, quantile)
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        pred = np.empty((len(self.models), N, H, W, 2), dtype=np.float32)
        for bi, s in enumerate(range(0, N, batch)):
            nb = min(batch, N - s)
            for k in range(len(self.models)):
                pred[k, s:s + nb] = outs[bi][k].reshape(nb, H, W, -1)[..., :2].cpu().numpy()
        nn.check()
        if screened is not None:
            mean, dis, rerun = screened
            return sec, pred, (mean.reshape(N, H, W).cpu().numpy().astype(np.float64), dis.cpu().numpy(),
                               rerun.cpu().numpy())
        return sec, pred

    @staticmethod
    def screen_device(pred0: torch.Tensor, threshold_m: float, quantile: float = 0.99):
        """``screen`` on the device: ``pred0`` [models, N, cells] is the networks' first output
        (log-depth); returns the mean peak depth [m] [N, cells], each member's disagreement
        (the ``quantile`` over its cells of the across-model spread of peak depth) and the
        rerun mask, all on the device."""
        t = pred0.float().clamp(0.0, float(np.log1p(MAX_DEPTH_M / DEPTH_SCALE_M)))
        depth = torch.expm1(t) * DEPTH_SCALE_M
        mean = depth.mean(dim=0)
        spread = depth.amax(dim=0) - depth.amin(dim=0)
        dis = torch.quantile(spread, quantile, dim=1)
        return mean, dis, dis > threshold_m

    @staticmethod
    def screen(pred: np.ndarray, threshold_m: float = 0.05, quantile: float = 0.99):
        """Mean predicted peak depth [m] per member map; each member's disagreement, the
        ``quantile`` over its cells of the across-model spread (max - min) of peak depth;
        and the members to rerun (disagreement above ``threshold_m``)."""
        depth = decode_depth_m(pred[..., 0])           # [models, N, H, W]
        mean = depth.mean(axis=0)
        spread = (depth.max(axis=0) - depth.min(axis=0)).reshape(depth.shape[1], -1)
        dis = np.quantile(spread, quantile, axis=1)
        return mean, dis, dis > threshold_m


def make_members(n: int, seed: int, size: int, **kw):
    from .synthetic import ensemble_member
    return [ensemble_member(i, seed=seed, lo=size, hi=size, **kw) for i in range(n)]


def dataset(cases, sol: SolveResult):
    X = np.stack([member_inputs(c) for c in cases])
    TW = [member_targets(d, a, c.params["routing_time"]) for c, d, a in zip(cases, sol.dmax_mm, sol.arrival_min)]
    return X, np.stack([t for t, _ in TW]), np.stack([w for _, w in TW])


def study(n_train: int = 4096, n_test: int = 1024, size: int = 256, epochs: int = 10, batch: int = 16,
          lr: float = 1e-3, seed: int = 7, n_fp64: int = 64, threshold_m: float = 0.05, log=None,
          member_kw: dict | None = None, screen_kinds=("rain",)) -> dict:
    """Trains the screening ensemble on solver output and measures it on held-out members:
    members/h of screening (inference + device-side disagreement screen + solver reruns of the
    flagged members) against the plain batched solver on the same members, overall and per
    member kind, and peak-depth errors against the FP64 solver on a subset.  Members whose kind
    is not in ``screen_kinds`` go to the solver without being screened: breach flows depend at
    metre scale on the time-step sequence itself (FP32 and FP64 solves of one breach member
    differ by up to 2 m in peak depth), so no network is held to 1 cm on them."""
    log = log or (lambda s: None)
    mk = dict(member_kw or {})
    t0 = time.perf_counter()
    train = make_members(n_train, seed, size, **mk)
    test = make_members(n_test, seed + 1, size, **mk)
    log(f"members generated in {time.perf_counter() - t0:.1f} s")
    sol_tr = solve_members(train)
    X, T, Wt = dataset(train, sol_tr)
    log(f"training set solved: {sol_tr.seconds:.2f} s device, {sol_tr.cell_updates / sol_tr.seconds / 1e9:.1f} GCUPS")
    scr = Screener(3, seed=seed)
    t1 = time.perf_counter()
    hist = scr.fit(X, T, Wt, epochs=epochs, batch=batch, lr=lr, seed=seed, log=log)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    sol_te = solve_members(test)
    Xte, Tte, Wte = dataset(test, sol_te)
    kinds = np.array([c.meta.get("kind", "") for c in test])
    screened_kind = np.isin(kinds, list(screen_kinds))
    t_inf, pred, (mean, dis, rerun_net) = scr.predict_timed(Xte[screened_kind], batch=32, threshold_m=threshold_m)
    rerun = np.ones(n_test, dtype=bool)          # unscreened kinds go to the solver
    rerun[screened_kind] = rerun_net
    mean_all = np.zeros((n_test,) + Xte.shape[1:3])
    mean_all[screened_kind] = mean
    mean = mean_all
    dis_all = np.full(n_test, np.inf)
    dis_all[screened_kind] = dis
    dis = dis_all
    idx = np.flatnonzero(rerun)
    t_rerun = solve_members([test[i] for i in idx]).seconds if idx.size else 0.0
    solver_mph = n_test / sol_te.seconds * 3600
    screened_mph = n_test / (t_inf + t_rerun) * 3600
    # the screened kinds on their own: plain solver on them against inference + their reruns
    sub = np.flatnonzero(screened_kind)
    sub_rerun = [i for i in sub if rerun[i]]
    t_sub_solver = solve_members([test[i] for i in sub]).seconds if sub.size else 0.0
    t_sub_rerun = solve_members([test[i] for i in sub_rerun]).seconds if sub_rerun else 0.0
    truth32 = np.stack([peak_m(d) for d in sol_te.dmax_mm])
    err32 = np.abs(mean - truth32).reshape(n_test, -1).max(axis=1)
    err32_sub = err32[screened_kind]
    # without training: an untrained ensemble of the same shape, on the same members
    # on the screened members (the networks' predictions exist for them only)
    k0 = min(int(sub.size), 64)
    _, pred0 = Screener(3, seed=seed + 999).predict_timed(Xte[sub[:k0]], batch=32)
    mean0 = decode_depth_m(pred0[..., 0]).mean(axis=0)
    err0 = np.abs(mean0 - truth32[sub[:k0]]).reshape(k0, -1).max(axis=1)
    # held-out loss of the training objective (ensemble-mean prediction), trained vs not
    held = lambda pr: float(np.mean(Wte[sub[:k0]] * (pr.mean(axis=0)[:k0] - Tte[sub[:k0]]) ** 2))
    loss_trained, loss_untrained = held(pred), held(pred0)
    wet = (truth32 > 0.01) & screened_kind[:, None, None]
    rms_wet = float(np.sqrt(np.mean((mean - truth32)[wet] ** 2))) if wet.any() else 0.0
    # FP64 solver on a subset of the held-out members
    k = min(n_fp64, n_test)
    sol64 = solve_members(test[:k], precision="fp64")
    truth64 = np.stack([peak_m(d) for d in sol64.dmax_mm])
    acc = ~rerun[:k]
    final = np.where(acc[:, None, None], mean[:k], truth32[:k])
    err_final = np.abs(final - truth64).reshape(k, -1).max(axis=1)
    sk = screened_kind[:k]
    err_sur64 = np.abs(mean[:k] - truth64).reshape(k, -1).max(axis=1)[sk] if sk.any() else np.zeros(1)
    err_solver32 = np.abs(truth32[:k] - truth64).reshape(k, -1).max(axis=1)
    q = lambda a, p: float(np.quantile(a, p))
    return dict(
        n_train=n_train, n_test=n_test, size=size, epochs=epochs, batch=batch,
        train_seconds=t_train, final_loss=[float(v) for v in hist[-1]],
        solver_seconds=sol_te.seconds, solver_gcups=sol_te.cell_updates / sol_te.seconds / 1e9,
        solver_members_per_h=solver_mph,
        inference_seconds=t_inf, rerun_members=int(idx.size), rerun_seconds=t_rerun,
        screened_members_per_h=screened_mph, speedup=screened_mph / solver_mph,
        screen_kinds=list(screen_kinds), screened_subset=dict(
            members=int(sub.size), rerun=len(sub_rerun),
            solver_members_per_h=sub.size / t_sub_solver * 3600 if t_sub_solver > 0 else None,
            screened_members_per_h=sub.size / (t_inf + t_sub_rerun) * 3600 if sub.size else None,
            speedup=(t_sub_solver / (t_inf + t_sub_rerun)) if sub.size else None,
            peak_err_vs_fp32_solver_m=dict(median=q(err32_sub, 0.5), p90=q(err32_sub, 0.9)) if sub.size else None),
        disagreement_m=dict(p50=q(dis, 0.5), p90=q(dis, 0.9)),
        peak_err_vs_fp32_solver_m=dict(median=q(err32, 0.5), p90=q(err32, 0.9)),
        untrained_peak_err_m=dict(median=q(err0, 0.5), p90=q(err0, 0.9)),
        heldout_loss=dict(trained=loss_trained, untrained=loss_untrained),
        peak_rms_wet_cells_m=rms_wet,
        rerun_by_kind={kd: [int(np.sum(rerun & (kinds == kd))), int(np.sum(kinds == kd))] for kd in np.unique(kinds)},
        fp64_subset=k, accepted_in_subset=int(acc.sum()),
        screened_peak_err_vs_fp64_m=dict(median=q(err_final, 0.5), max=float(err_final.max())),
        surrogate_peak_err_vs_fp64_m=dict(median=q(err_sur64, 0.5), p90=q(err_sur64, 0.9)),
        solver32_peak_err_vs_fp64_m=dict(max=float(err_solver32.max())),
        within_1cm_share=float(np.mean(err_final <= 0.01)),
    )
