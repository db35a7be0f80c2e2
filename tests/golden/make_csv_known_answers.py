"""Extract the reference's published known answers into a small fixture.

Reads the reference's merged summary CSV
(ring_cx_pipeline_vs_original_structed_vs_inversecuQuantum/
 originstructed_vs_cuquantum_8to24q_2layers_summary_merged.csv) and writes
csv_known_answers.json: for each qubit count, the final energy after 20
plain gradient-descent steps (stepsize 0.08, seed 7, init 0.3*N(0,1), h=1,
L=2) from both of the reference's GPU strategies.

Run with the reference checkout at REF (default: a directory "reference"
beside this repository's checkout):
    python tests/golden/make_csv_known_answers.py
"""

from __future__ import annotations

import csv
import json
import os
from pathlib import Path

REF = Path(os.environ.get("REF", str(Path(__file__).resolve().parents[3] / "reference")))
CSV = (
    REF
    / "ring_cx_pipeline_vs_original_structed_vs_inversecuQuantum"
    / "originstructed_vs_cuquantum_8to24q_2layers_summary_merged.csv"
)


def main() -> None:
    rows = {}
    with CSV.open(newline="") as fh:
        for row in csv.DictReader(fh):
            if row["status"] != "ok":
                continue
            n = int(row["num_qubits"])
            rows.setdefault(str(n), {})[row["method"]] = float(row["final_energy"])
    out = {
        "source": "reference CSV originstructed_vs_cuquantum_8to24q_2layers_summary_merged.csv, column final_energy",
        "protocol": {"layers": 2, "field": 1.0, "steps": 20, "stepsize": 0.08, "seed": 7, "init_scale": 0.3},
        "final_energy": rows,
    }
    dst = Path(__file__).with_name("csv_known_answers.json")
    dst.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {dst} ({len(rows)} qubit counts)")


if __name__ == "__main__":
    main()
