"""Generates tests/golden/default_run_seed42.json with the CPU oracle.

    python tests/golden/make_golden.py

The reference default run (128x128x64, Winogradsky priming, 3 x 30 starter
cells) on the oracle's seeded RNG (seed 42), fingerprinted at ticks 1, 10,
100, 300 and 1000: population, division and death totals, SHA-256 of the
cell positions and of the lineage ids in cell-vector order, and the per-species
FP64 sums of the field.  About four minutes on 8 cores (the oracle's cell
loop is sequential, as the reference's is).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402


def fingerprint(cells: np.ndarray, field: np.ndarray, stats: dict) -> dict:
    return {
        "tick": stats["tick"],
        "population": stats["population"],
        "total_divisions": stats["total_divisions"],
        "total_deaths": stats["total_deaths"],
        "positions_sha256": hashlib.sha256(np.ascontiguousarray(cells["pos"]).tobytes()).hexdigest(),
        "lineage_sha256": hashlib.sha256(np.ascontiguousarray(cells["lineage_id"]).tobytes()).hexdigest(),
        "field_species_sums": [float(v) for v in field.reshape(-1, 12).astype(np.float64).sum(0)],
    }


def main() -> int:
    oracle.set_threads(os.cpu_count() or 1)
    w = oracle.World((128, 128, 64), seed=42, seed_count=30)
    out = {"workload": "reference default run 128x128x64, seed_count 30, oracle RNG seed 42", "ticks": []}
    for t in (1, 10, 100, 300, 1000):
        w.tick(t - w.stats()["tick"])
        out["ticks"].append(fingerprint(w.cells(), w.field(), w.stats()))
        print(out["ticks"][-1]["tick"], out["ticks"][-1]["population"], flush=True)
    with open(os.path.join(HERE, "default_run_seed42.json"), "w") as f:
        json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
