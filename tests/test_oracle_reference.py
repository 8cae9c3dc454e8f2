"""CPU oracle pinned against the reference's own tests and fixtures, and
cross-checked against the independent numpy restatement.

Reference tests restated here:
  crates/marl-field/src/field.rs:270-289  occupied_voxel_is_copied_unchanged
  crates/marl-field/src/field.rs:291-312  deterministic_diffusion_stays_finite_and_nonnegative
  crates/marl-gpu/tests/gpu_diffusion.rs:81-150  4 occupancy patterns, substeps 1/2/10,
      max abs error <= 1e-4 between two implementations (here: C++ oracle vs the
      numpy restatement of the WGSL shader; they agree bit-for-bit)
  crates/marl-config/src/lib.rs:108-168  SimulationConfig defaults
"""
import numpy as np
import pytest

from conftest import deterministic_field, occupancy_patterns, wave_field

FULL = (128, 128, 64)  # the reference's compile-time grid


def test_default_params_match_reference(oracle_mod):
    p = oracle_mod.default_params()
    assert p.dt == 1.0 and p.diffusion_substeps == 10
    np.testing.assert_array_equal(np.array(list(p.d_voxel), np.float32),
                                  np.array([0.0, 1.5, 1.0, 1.2, 0.8, 0.5, 0.5, 0.1, 0.3, 0.3, 0.3, 0.3], np.float32))
    np.testing.assert_array_equal(np.array(list(p.lambda_decay), np.float32),
                                  np.array([0.0, 0.01, 0.01, 0.005, 0.03, 0.05, 0.05, 0.002, 0.01, 0.01, 0.01, 0.01],
                                           np.float32))
    assert (p.source_rate_oxidant, p.source_rate_carbon, p.source_rate_reductant) == pytest.approx((0.4, 0.15, 0.5))
    assert p.c_max == 10.0 and p.alpha_eps == pytest.approx(0.8) and p.k_eps == 2.0
    assert p.cell_absorption == pytest.approx(0.3) and p.chemical_absorption == pytest.approx(0.05)
    assert p.light_floor == np.float32(1e-7) and p.active_reaction_threshold == np.float32(1e-9)
    assert p.division_neighbor_distance == 2 and p.seed_margin == 5 and p.boundary_prime_layers == 2


def test_occupied_voxel_is_copied_unchanged(oracle_mod):
    p = oracle_mod.default_params()
    p.diffusion_substeps = 1
    X, Y, Z = FULL
    f = deterministic_field(FULL)
    occ = np.zeros((Z, Y, X), np.uint8)
    occ[Z // 2, Y // 2, X // 2] = 1
    before = f[Z // 2, Y // 2, X // 2].copy()
    oracle_mod.diffuse(f, occ, FULL, p, 1)
    np.testing.assert_array_equal(f[Z // 2, Y // 2, X // 2], before)


def test_deterministic_diffusion_stays_finite_and_nonnegative(oracle_mod):
    p = oracle_mod.default_params()
    p.diffusion_substeps = 1
    f = deterministic_field(FULL)
    occ = np.zeros(FULL[::-1], np.uint8)
    oracle_mod.diffuse(f, occ, FULL, p, 1)
    assert np.isfinite(f).all()
    assert (f >= 0).all()


@pytest.mark.parametrize("pattern", ["empty", "center", "boundary_adjacent", "dense_cluster"])
@pytest.mark.parametrize("substeps", [1, 2, 10])
def test_oracle_matches_wgsl_restatement(oracle_mod, pattern, substeps):
    import ref_numpy

    dims = (48, 40, 24)
    p = oracle_mod.default_params()
    f0 = wave_field(dims)
    occ = occupancy_patterns(dims)[pattern]
    a = f0.copy()
    oracle_mod.diffuse(a, occ, dims, p, substeps)
    b = ref_numpy.diffuse_tick(f0, occ, p, substeps)
    assert np.abs(a - b).max() <= 1e-4  # the reference's own tolerance
    np.testing.assert_array_equal(a, b)  # and in fact bit-identical


def test_oracle_matches_wgsl_restatement_full_grid(oracle_mod):
    import ref_numpy

    p = oracle_mod.default_params()
    f0 = wave_field(FULL)
    occ = occupancy_patterns(FULL)["dense_cluster"]
    a = f0.copy()
    oracle_mod.diffuse(a, occ, FULL, p, 2)
    np.testing.assert_array_equal(a, ref_numpy.diffuse_tick(f0, occ, p, 2))


def test_sources_match_restatement(oracle_mod):
    import ref_numpy

    dims = (16, 12, 8)
    p = oracle_mod.default_params()
    f = np.random.default_rng(1).random((8, 12, 16, 12), dtype=np.float32) * np.float32(10.0)
    a = f.copy()
    oracle_mod.sources(a, dims, p)
    b = f.copy()
    ref_numpy.sources(b, p)
    np.testing.assert_array_equal(a, b)
    assert (a[0, :, :, 1] <= 10.0).all() and (a[-1, :, :, 2] <= 10.0).all()


def test_light_matches_restatement(oracle_mod):
    import ref_numpy

    dims = (24, 20, 32)
    rng = np.random.default_rng(7)
    f = rng.random((32, 20, 24, 12), dtype=np.float32) * np.float32(3.0)
    occ = (rng.random((32, 20, 24)) < 0.1).astype(np.uint8)
    p = oracle_mod.default_params()
    a = oracle_mod.light(f, occ, dims, p)
    b = ref_numpy.light(f, occ, p)
    # exp implementations differ by at most an ulp per factor
    np.testing.assert_allclose(a, b, rtol=2e-6, atol=1e-12)
    assert (a[0] == p.surface_intensity).all()


def test_light_known_column(oracle_mod):
    """Beer-Lambert column by hand: I0 = 1, one cell at z=1, absorber a at z=2."""
    dims = (1, 1, 5)
    p = oracle_mod.default_params()
    f = np.zeros((5, 1, 1, 12), np.float32)
    f[2, 0, 0, 4] = 4.0
    occ = np.zeros((5, 1, 1), np.uint8)
    occ[1] = 1
    L = oracle_mod.light(f, occ, dims, p)[:, 0, 0]
    e_cell = np.float32(np.exp(np.float64(-np.float32(0.3))))
    e_abs = np.float32(np.exp(np.float64(np.float32(-0.05) * np.float32(4.0))))
    np.testing.assert_allclose(L, [1.0, 1.0, e_cell, e_cell * e_abs, e_cell * e_abs], rtol=1e-6)
    # floor to zero is absorbing
    f[2, 0, 0, 4] = 1000.0
    L = oracle_mod.light(f, occ, dims, p)[:, 0, 0]
    assert L[3] == 0.0 and L[4] == 0.0


def test_cell_tick_matches_restatement(oracle_mod):
    import ref_numpy
    from helpers import random_cells

    rng = np.random.default_rng(3)
    p = oracle_mod.default_params()
    cells = random_cells((8, 8, 8), 64, rng)
    for c in cells:
        ext = rng.random(12, dtype=np.float32)
        light = np.float32(rng.random())
        c1, d1, e1 = oracle_mod.cell_tick(c, ext, light, p)
        c2, d2, e2 = ref_numpy.cell_tick(c, ext, light, p)
        np.testing.assert_array_equal(c1["internal"], c2["internal"])
        np.testing.assert_array_equal(d1, d2)
        assert e1 == e2
        assert c1["prep_remaining"] == c2["prep_remaining"] and c1["quiescent"] == c2["quiescent"]


def test_cell_tick_known_answer(oracle_mod):
    """One transporter, no reactions: values by hand."""
    from marl_cuda import CELL_DTYPE

    p = oracle_mod.default_params()
    c = oracle_mod.make_starter(0, [1, 1, 1], 1)
    rs = c["ruleset"]
    rs["reactions"]["v_max"] = 0.0
    rs["transport"]["uptake_rate"] = 0.0
    rs["transport"]["secrete_rate"] = 0.0
    rs["effectors"]["rate"] = 0.0
    rs["transport"][0] = (0.6, 0.0, 3, 3, [0, 0])
    c["internal"] = 0.0
    c["internal"][0] = 1.0
    ext = np.zeros(12, np.float32)
    ext[3] = 0.5
    out, d, ev = oracle_mod.cell_tick(np.array(c, CELL_DTYPE), ext, 0.25, p)
    f = np.float32
    uptake = f(0.6) * f(0.5) / (f(1.0) + f(0.5))
    assert out["internal"][3] == uptake  # 0.2
    assert d[3] == (f(0.0) - uptake) * f(1.0)
    assert out["internal"][15] == f(0.25)  # light slot
    assert out["internal"][0] == f(1.0) * (f(1.0) - f(0.12) * f(1.0) * f(1.0))  # maintenance, no active rxns
    assert ev == 0 and out["age"] == c["age"] + 1


def test_sequential_order_matters(oracle_mod):
    """Two cells sharing one empty voxel: the second reads the first's deltas."""
    from helpers import random_cells

    dims = (3, 1, 1)
    rng = np.random.default_rng(11)
    cells = random_cells(dims, 2, rng, positions=np.array([[0, 0, 0], [2, 0, 0]]))
    f = np.full((1, 1, 3, 12), 0.5, np.float32)
    light = np.ones((1, 1, 3), np.float32)
    p = oracle_mod.default_params()
    fa, ca, _ = oracle_mod.cell_phase(f, light, cells, dims, p)
    fb, cb, _ = oracle_mod.cell_phase(f, light, cells[::-1].copy(), dims, p)
    assert not np.array_equal(fa, fb)  # order changes the result (Gauss-Seidel)
    # the first cell of the loop sees the untouched field: same as ticking it alone
    solo_f, solo_c, _ = oracle_mod.cell_phase(f, light, cells[:1].copy(), dims, p)
    np.testing.assert_array_equal(ca[0]["internal"], solo_c[0]["internal"])


def test_cell_phase_matches_restatement(oracle_mod):
    import ref_numpy
    from helpers import clustered_positions, random_cells, random_field

    dims = (10, 9, 8)
    rng = np.random.default_rng(5)
    pos = clustered_positions(dims, 0.3, rng, 1, 2)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    f = random_field(dims, rng)
    light = rng.random((8, 9, 10), dtype=np.float32)
    p = oracle_mod.default_params()
    fa, ca, ea = oracle_mod.cell_phase(f, light, cells, dims, p)
    fb, cb, eb = ref_numpy.cell_phase(f, light, cells, dims, p)
    np.testing.assert_array_equal(fa, fb)
    np.testing.assert_array_equal(ca["internal"], cb["internal"])
    np.testing.assert_array_equal(ea, eb)


def test_fate_swap_remove_and_births(oracle_mod):
    """lib.rs:219-277: deaths swap_remove'd back to front, births appended."""
    from helpers import random_cells

    dims = (12, 12, 12)
    rng = np.random.default_rng(2)
    cells = random_cells(dims, 6, rng, positions=np.array([[1, 1, 1], [5, 5, 5], [9, 9, 9], [1, 9, 1], [9, 1, 9],
                                                          [5, 1, 5]]))
    w = oracle_mod.World(dims, seed=9, seed_count=None)
    w.set_cells(cells)
    ev = np.array([2, 0, 2, 0, 0, 0], np.int32)  # deaths of 0 and 2
    w.fate(ev)
    out = w.cells()
    # swap_remove(2): [0,1,5,3,4]; swap_remove(0): [4,1,5,3]
    assert [tuple(c["pos"]) for c in out] == [tuple(cells[i]["pos"]) for i in (4, 1, 5, 3)]
    occ = w.occupancy()
    assert occ.sum() == 4 and occ[1, 1, 1] == 0 and occ[9, 9, 9] == 0


def test_world_seeding_bands(oracle_mod):
    """seed_cells depth bands at Z=64: photo [0,1), chemo [25,41), anaerobe [38,57)."""
    w = oracle_mod.World((128, 128, 64), seed=42, seed_count=30)
    c = w.cells()
    assert len(c) == 90
    z = c["pos"][:, 2]
    st = c["starter_type"]
    assert (z[st == 0] == 0).all()
    assert ((z[st == 1] >= 25) & (z[st == 1] < 41)).all()
    assert ((z[st == 2] >= 38) & (z[st == 2] < 57)).all()
    assert (c["pos"][:, :2] >= 5).all() and (c["pos"][:, :2] < 123).all()
    f = w.field()
    assert (f[:2, :, :, 1] == np.float32(0.5)).all() and (f[-2:, :, :, 2] == np.float32(0.5)).all()
