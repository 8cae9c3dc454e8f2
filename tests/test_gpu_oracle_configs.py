"""Parity against the CPU oracle at the benchmark configurations' own sizes.

- Batched ensemble (four uneven grids of the 64-run ensemble, 64x64x32 to
  128x128x96, the ensemble's seeds): every run of one marl_batch against an
  oracle World with the same seed, tick by tick (crates/marl-sim/src/lib.rs:
  160-277): population, positions and lineages exact, internals within 1e-4,
  with fate events exercised; host fate and device fate.
- Field microbenchmark at 256x256x128 (8.4M voxels): sources fused into the
  first of three substeps, additive and Dirichlet, bit-exact against the
  oracle (crates/marl-field/src/field.rs:107-250); the light scan within 1e-5
  relative (crates/marl-field/src/light.rs:29-59).
- Cell microbenchmark: one cell phase over the full 1,000,000-cell table on
  256x256x128, bit-exact against the oracle's sequential loop
  (crates/marl-sim/src/lib.rs:206-217).
- Error against the FP64 oracle, per phase on identical inputs: diffusion,
  light and the cell phase of the reference default run at tick 1 and at
  tick 100, asserted within 1e-5 relative (absolute floor 1e-6) and printed.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Runs i = 0, 16, 32, 48 of the 64-run ensemble: grid i // 16, seed i.
ENSEMBLE_RUNS = [((64, 64, 32), 0), ((96, 96, 48), 16), ((128, 128, 64), 32), ((128, 128, 96), 48)]


@pytest.mark.parametrize("device_fate", [False, True])
def test_batch_matches_oracle_runs(marl, oracle_mod, device_fate):
    p = marl.default_params()
    ticks = 30
    b = marl.Batch(ENSEMBLE_RUNS, p, seed_count=30, cell_capacity=1 << 16)
    worlds = [oracle_mod.World(dims, p, seed=seed, seed_count=30) for dims, seed in ENSEMBLE_RUNS]
    if device_fate:
        b.set_device_fate(True)
        for w in worlds:
            w.set_fate_mode(1)  # per-division streams keyed by (run seed, tick, parent)
    for r, w in enumerate(worlds):
        assert b.cells(r).tobytes() == w.cells().tobytes()
    for t in range(ticks):
        b.step(1)
        for r, w in enumerate(worlds):
            w.tick(1)
            bs, ws = b.stats(r), w.stats()
            assert (bs["population"], bs["total_divisions"], bs["total_deaths"]) == (
                ws["population"], ws["total_divisions"], ws["total_deaths"]), (t, r, bs, ws)
            gc, wc = b.cells(r), w.cells()
            np.testing.assert_array_equal(gc["pos"], wc["pos"])
            np.testing.assert_array_equal(gc["lineage_id"], wc["lineage_id"])
            assert gc["ruleset"].tobytes() == wc["ruleset"].tobytes()
            np.testing.assert_allclose(gc["internal"], wc["internal"], rtol=1e-4, atol=1e-5)
    events = 0
    for r, w in enumerate(worlds):
        np.testing.assert_allclose(b.field(r), w.field(), rtol=1e-4, atol=1e-5)
        s = b.stats(r)
        events += s["total_divisions"] + s["total_deaths"]
    assert events > 0, "no fate events: the edit path was not exercised"
    b.close()


def micro_context(marl, p, occ):
    import workloads  # noqa: F401  (sys.path set by conftest)

    z, y, x = np.nonzero(occ)
    walls = np.zeros(len(x), marl.CELL_DTYPE)  # occupancy only
    walls["pos"] = np.stack([x, y, z], 1).astype(np.uint16)
    dims = (occ.shape[2], occ.shape[1], occ.shape[0])
    ctx = marl.Context(dims, p, cell_capacity=len(walls))
    ctx.upload_cells(walls)
    return ctx


@pytest.mark.parametrize("mode", ["additive", "dirichlet"])
def test_field_microbench_full_size(marl, oracle_mod, mode):
    import workloads

    dims = workloads.MICRO_DIMS
    field, occ = workloads.field_microbench()
    p = marl.default_params()
    p.source_mode = 0 if mode == "additive" else 1
    ctx = micro_context(marl, p, occ)
    ctx.upload_field(field)
    ctx.diffuse(3, fuse_sources=True)
    got = ctx.download_field()
    ctx.light_update()
    got_light = ctx.download_light()
    ctx.close()
    want = field.copy()
    oracle_mod.sources(want, dims, p)
    oracle_mod.diffuse(want, occ, dims, p, 3)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    want_light = oracle_mod.light(want, occ, dims, p)
    np.testing.assert_allclose(got_light, want_light, rtol=1e-5, atol=1e-6)


def test_cell_microbench_full_size(marl, oracle_mod):
    import workloads

    dims = workloads.MICRO_DIMS
    X, Y, Z = dims
    field, _ = workloads.field_microbench()
    cells = workloads.cell_microbench()
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=len(cells))
    ctx.upload_field(field)
    ctx.upload_cells(cells)
    ctx.light_update()  # one light scan on the cells' occupancy
    light = ctx.download_light()
    ev = ctx.cell_phase()
    got_field, got_cells = ctx.download_field(), ctx.download_cells()
    ctx.close()
    want_field, want_cells, want_ev = oracle_mod.cell_phase(field, light, cells, dims, p)
    assert np.array_equal(got_field.view(np.uint32), want_field.view(np.uint32))
    assert np.array_equal(got_cells["internal"].view(np.uint32), want_cells["internal"].view(np.uint32))
    np.testing.assert_array_equal(got_cells["prep_remaining"], want_cells["prep_remaining"])
    np.testing.assert_array_equal(got_cells["quiescent"], want_cells["quiescent"])
    np.testing.assert_array_equal(got_cells["age"], want_cells["age"])
    np.testing.assert_array_equal(ev.astype(np.int32), want_ev)


def fp64_report(name, got, want64, rtol=1e-5, atol=1e-6):
    """Largest error of an FP32 result against the FP64 oracle, as a fraction
    of the allowed rtol*|want| + atol, and the largest relative error where
    |want| >= 1e-3."""
    got = np.asarray(got, np.float64)
    d = np.abs(got - want64)
    ratio = float((d / (rtol * np.abs(want64) + atol)).max()) if d.size else 0.0
    big = np.abs(want64) >= 1e-3
    rel = float((d[big] / np.abs(want64[big])).max()) if big.any() else 0.0
    print(f"  {name:<24} max rel err {rel:.3e} (|v| >= 1e-3), max err / tolerance {ratio:.3f}")
    return ratio


@pytest.mark.parametrize("tick", [1, 100])
def test_default_run_against_fp64_oracle(marl, oracle_mod, tick):
    """One tick of the reference default run (128x128x64, seed 42), phase by
    phase on identical FP32 inputs, against the FP64 oracle."""
    dims = (128, 128, 64)
    p = marl.default_params()
    eng = marl.Engine(dims, p, rng_seed=42, seed_count=30, cell_capacity=1 << 16)
    if tick > 1:
        eng.step(tick - 1)
    field0, cells = eng.field(), eng.cells()
    eng.close()
    ctx = marl.Context(dims, p, cell_capacity=max(len(cells), 1))
    ctx.upload_field(field0)
    ctx.upload_cells(cells)
    occ = ctx.download_occupancy()
    ctx.diffuse(p.diffusion_substeps, fuse_sources=True)
    field1 = ctx.download_field()
    ctx.light_update()
    light1 = ctx.download_light()
    ctx.cell_phase()
    field2, cells2 = ctx.download_field(), ctx.download_cells()
    ctx.close()

    print(f"\ntick {tick}, {len(cells)} cells, against the FP64 oracle:")
    r = [fp64_report("diffusion (10 substeps)", field1,
                     oracle_mod.diffuse_f64(field0, occ, dims, p, p.diffusion_substeps, apply_sources=True)),
         fp64_report("light", light1, oracle_mod.light_f64(field1, occ, dims, p))]
    f64, int64 = oracle_mod.cell_phase_f64(field1, light1, cells, dims, p)
    r.append(fp64_report("cell phase: field", field2, f64))
    r.append(fp64_report("cell phase: internals", cells2["internal"], int64))
    assert max(r) <= 1.0, r
