"""Generates the golden fixtures in this folder from the reference repository.

Run in the build container (the reference checkout is not present on GPU machines):

    python tests/golden/make_golden.py /path/to/HydroPol2D

* green_ampt_reference.csv -- the Green-Ampt analytical cumulative infiltration of case
  P1-INFIL-GA-001, produced by calling the reference's own generator
  Validation/scripts/phase1_reference_solutions.py (green_ampt_cumulative, :208-225) with the
  case parameters of green_ampt (:228-249): Ks = 1e-6 m/s, psi*dtheta = 0.055 m, 30-min samples.
* registry_metrics.json -- metrics of real runs of the current local-inertial code recorded
  in the reference's validation registry Validation/Phase1_Cases.csv (notes column of rows
  P1-HYDRO-LI-RITTER-001 and P1-HYDRO-LI-PLANE-001), parsed from that file.
"""
from __future__ import annotations

import csv
import importlib.util
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    spec = importlib.util.spec_from_file_location(
        "phase1_reference_solutions", ref / "Validation" / "scripts" / "phase1_reference_solutions.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    ks, psi_dtheta = 1.0e-6, 0.055
    rows = []
    for step in range(49):
        t = step * 1800.0
        rows.append({"time_s": t, "cumulative_infiltration_m": mod.green_ampt_cumulative(t, ks, psi_dtheta),
                     "Ks_m_s": ks, "psi_delta_theta_m": psi_dtheta})
    with open(HERE / "green_ampt_reference.csv", "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=list(rows[0]))
        w.writeheader()
        w.writerows(rows)

    reg = {}
    with open(ref / "Validation" / "Phase1_Cases.csv", newline="", encoding="utf-8") as f:
        for row in csv.DictReader(f):
            cid, note = row["case_id"], row["notes"]
            if cid == "P1-HYDRO-LI-RITTER-001":
                m = re.search(r"RMSE ([0-9.]+) m, relative L2 ([0-9.]+)", note)
                reg[cid] = {"rmse_m": float(m.group(1)), "relative_l2": float(m.group(2)), "note": note}
            elif cid == "P1-HYDRO-LI-PLANE-001":
                m = re.search(r"NSE ([0-9]+\.[0-9]+)", note)
                reg[cid] = {"nse": float(m.group(1)), "note": note}
    reg["source"] = "Validation/Phase1_Cases.csv (notes column)"
    (HERE / "registry_metrics.json").write_text(json.dumps(reg, indent=2) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/HydroPol2D")
    main(sys.argv[1])
