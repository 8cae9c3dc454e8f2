"""The reference default run against committed fingerprints of the CPU oracle
(tests/golden/default_run_seed42.json, made by tests/golden/make_golden.py).

CPU: the oracle still reproduces its own fingerprints at ticks 1 and 10.
GPU: the engine, advanced through the C ABI to ticks 1, 10, 100, 300 and 1000,
has the same population, division and death totals, cell positions and
lineage ids (hashed, in cell-vector order) as the oracle, and per-species
field sums within 1e-5 relative (the light scan's exp is within 1e-5, not
bit-exact).
"""
import hashlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "default_run_seed42.json")
DIMS = (128, 128, 64)


def load():
    with open(GOLDEN) as f:
        return json.load(f)["ticks"]


def check(fp, cells, field, stats):
    assert stats["population"] == fp["population"], fp["tick"]
    assert stats["total_divisions"] == fp["total_divisions"], fp["tick"]
    assert stats["total_deaths"] == fp["total_deaths"], fp["tick"]
    assert hashlib.sha256(np.ascontiguousarray(cells["pos"]).tobytes()).hexdigest() == fp["positions_sha256"]
    assert hashlib.sha256(np.ascontiguousarray(cells["lineage_id"]).tobytes()).hexdigest() == fp["lineage_sha256"]
    sums = field.reshape(-1, 12).astype(np.float64).sum(0)
    np.testing.assert_allclose(sums, fp["field_species_sums"], rtol=1e-5, atol=1e-6)


def test_oracle_reproduces_golden(oracle_mod):
    oracle_mod.set_threads(oracle_mod.max_threads())
    w = oracle_mod.World(DIMS, seed=42, seed_count=30)
    for fp in load():
        if fp["tick"] > 10:
            break
        w.tick(fp["tick"] - w.stats()["tick"])
        check(fp, w.cells(), w.field(), w.stats())


@pytest.mark.gpu
def test_engine_matches_golden_to_tick_1000(marl):
    e = marl.Engine(DIMS, marl.default_params(), rng_seed=42, seed_count=30, cell_capacity=1 << 20)
    for fp in load():
        e.step(fp["tick"] - e.stats()["tick"])
        check(fp, e.cells(), e.field(), e.stats())
