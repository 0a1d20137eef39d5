"""Pins of the oracle against the reference's own validation evidence (no GPU).

* The validation registry records metrics of real runs of the current local-inertial code
  (tests/golden/registry_metrics.json, parsed from Validation/Phase1_Cases.csv): Ritter
  dam-break RMSE 0.182 m and relative L2 0.384, tilted plane NSE 0.998.  The restatements must
  reproduce them to the printed precision.
* The driver's acceptance gates (run_local_inertial_ca_hydrodynamics_validation.m:113, :197):
  plane mass < 0.1 %, NSE > 0.70, relative L2 < 0.45; V-tilt mass < 0.1 %, symmetry RMSE < 1e-8 m,
  channel wet.
* Green-Ampt: the explicit capacity form converges to the analytical cumulative infiltration of
  P1-INFIL-GA-001 (tests/golden/green_ampt_reference.csv).
"""
import csv
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import literal as L
from tests import validation_cases as V

GOLD = Path(__file__).resolve().parent / "golden"
REG = json.loads((GOLD / "registry_metrics.json").read_text())


def kernel_form_step(case_fn, precision):
    import oracle
    c = case_fn()
    ny, nx = c["z"].shape
    o = oracle.KernelFormOracle(ny, nx, c["dx"], precision, outlet_type=1, slope_outlet=c["slope"])
    return V.SurfaceStep(o, c["z"], c["n"], c["dx"], c["rows"], c["cols"], c["slope"])


def literal_step(case_fn):
    c = case_fn()
    return V.LiteralStep(c["z"], c["n"], c["dx"], c["rows"], c["cols"], c["slope"])


# ---------------------------------------------------------------- registry metrics
def test_literal_ritter_reproduces_registry():
    m = V.run_ritter(literal_step(V.ritter_case))
    reg = REG["P1-HYDRO-LI-RITTER-001"]
    assert round(m["rmse"], 3) == reg["rmse_m"]
    assert round(m["rel_l2"], 3) == reg["relative_l2"]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_kernel_form_ritter_reproduces_registry(oracle_lib, precision):
    m = V.run_ritter(kernel_form_step(V.ritter_case, precision))
    reg = REG["P1-HYDRO-LI-RITTER-001"]
    assert abs(m["rmse"] - reg["rmse_m"]) < 1e-3
    assert abs(m["rel_l2"] - reg["relative_l2"]) < 1e-3


def test_literal_plane_reproduces_registry_and_gates():
    m = V.run_plane(literal_step(V.plane_case))
    assert round(m["nse"], 3) == REG["P1-HYDRO-LI-PLANE-001"]["nse"]
    assert m["mass_pct"] < 0.1 and m["nse"] > 0.70 and m["rel_l2"] < 0.45


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_kernel_form_plane_gates(oracle_lib, precision):
    m = V.run_plane(kernel_form_step(V.plane_case, precision))
    assert abs(m["nse"] - REG["P1-HYDRO-LI-PLANE-001"]["nse"]) < 1e-3
    assert m["mass_pct"] < 0.1 and m["rel_l2"] < 0.45


# ---------------------------------------------------------------- V-tilt symmetry / mass
def test_literal_vtilt_gates():
    m = V.run_vtilt(literal_step(V.vtilt_case))
    assert m["symmetry_rmse"] < 1e-8 and m["mass_pct"] < 0.1 and m["channel_depth"] > 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_kernel_form_vtilt_exact_symmetry(oracle_lib, precision):
    m = V.run_vtilt(kernel_form_step(V.vtilt_case, precision))
    assert m["symmetry_rmse"] == 0.0
    assert m["mass_pct"] < 0.1 and m["channel_depth"] > 0


# ---------------------------------------------------------------- Green-Ampt analytical
def _ga_reference():
    rows = list(csv.DictReader(open(GOLD / "green_ampt_reference.csv")))
    return np.array([float(r["time_s"]) for r in rows]), np.array([float(r["cumulative_infiltration_m"]) for r in rows])


def _ga_params(n=1):
    # Ks = 1e-6 m/s = 3.6 mm/h, psi * dtheta = 0.055 m (psi 220 mm, dtheta 0.25)
    return L.GAParams(ksat=np.full(n, 3.6), psi=np.full(n, 220.0), dtheta=np.full(n, 0.25),
                      Lu=np.full(n, 1e9), k_out=np.zeros(n), Tr=np.full(n, 1e9),
                      min_sm=np.full(n, np.finfo(float).eps), active=np.ones(n, bool))


def test_literal_green_ampt_converges_to_analytical():
    """Ponded column (0.1 mm kept on the surface) at dt = 0.5 s: cumulative infiltration
    against the analytical P1-INFIL-GA-001 curve (2 % from 30 min on, up to 6 h)."""
    t_ref, F_ref = _ga_reference()
    p = _ga_params()
    I = np.full(1, np.finfo(float).eps)
    T = np.full(1, 1e9)
    ts = 0.5 / 60
    F = 0.0
    checks = {}
    for k in range(1, int(6 * 3600 / 0.5) + 1):
        d = np.full(1, 0.1)
        dn, I, T, f = L.green_ampt_infiltration(d, I, T, ts, p, 1.0)
        F += f[0] * ts / 60 / 1000
        t = k * 0.5
        if t % 1800 == 0:
            checks[t] = F
    for t, Fm in checks.items():
        Fa = F_ref[np.where(t_ref == t)[0][0]]
        assert abs(Fm - Fa) / Fa < 0.02, (t, Fm, Fa)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_kernel_form_green_ampt_converges_to_analytical(oracle_lib, precision):
    import oracle
    t_ref, F_ref = _ga_reference()
    o = oracle.KernelFormOracle(1, 1, 1.0, precision, flag_infiltration=1)
    o.upload_static(np.zeros((1, 1)), np.full((1, 1), 0.03), [], [])
    o.set_soil(np.zeros((1, 1), np.uint8), [3.6], [220.0], [0.25], [1e9], [0.0], [1e9], [np.finfo(float).eps])
    o.set_state(np.full((1, 1), 1e-3), None, np.full((1, 1), np.finfo(float).eps))
    ts = 0.5 / 60
    for k in range(1, int(3 * 3600 / 0.5) + 1):
        o.set_depth(np.full((1, 1), 0.1))
        o.hydrology_step(ts)
        t = k * 0.5
        if t % 1800 == 0:
            Fm = float(o.download_native("I")[0, 0])
            Fa = F_ref[np.where(t_ref == t)[0][0]]
            assert abs(Fm - Fa) / Fa < 0.02, (t, Fm, Fa)
