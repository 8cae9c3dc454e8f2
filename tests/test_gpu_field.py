"""GPU parity of the field kernels against the CPU oracle, through the C ABI.

Diffusion and boundary sources are compared bit-for-bit (the reference's own
GPU test, crates/marl-gpu/tests/gpu_diffusion.rs:60-111, allows max abs 1e-4).
Light is compared within 1e-5 relative error (floor 1e-6 absolute); the
fraction of bit-identical voxels is asserted too.
"""
import numpy as np
import pytest

from conftest import occupancy_patterns, wave_field

pytestmark = pytest.mark.gpu

FULL = (128, 128, 64)
LIGHT_RTOL = 1e-5
LIGHT_ATOL = 1e-6


def ctx_with(marl, dims, params=None, cells=None, field=None, cap=4096):
    ctx = marl.Context(dims, params, cell_capacity=cap)
    if field is not None:
        ctx.upload_field(field)
    if cells is not None:
        ctx.upload_cells(cells)
    return ctx


def cells_at(marl, occ):
    """Cell records at the occupied voxels of a [z,y,x] mask (only positions matter for the field)."""
    z, y, x = np.nonzero(occ)
    c = np.zeros(len(x), marl.CELL_DTYPE)
    c["pos"] = np.stack([x, y, z], 1).astype(np.uint16)
    return c


@pytest.mark.parametrize("pattern", ["empty", "center", "boundary_adjacent", "dense_cluster"])
@pytest.mark.parametrize("substeps", [1, 2, 10])
def test_diffusion_reference_patterns(marl, oracle_mod, pattern, substeps):
    p = marl.default_params()
    p.diffusion_substeps = substeps
    f0 = wave_field(FULL)
    occ = occupancy_patterns(FULL)[pattern]
    ctx = ctx_with(marl, FULL, p, cells_at(marl, occ), f0)
    ctx.diffuse(substeps)
    gpu = ctx.download_field()
    cpu = f0.copy()
    oracle_mod.diffuse(cpu, occ, FULL, p, substeps)
    assert np.abs(gpu - cpu).max() <= 1e-4
    np.testing.assert_array_equal(gpu, cpu)


@pytest.mark.parametrize("dims", [(37, 21, 13), (16, 16, 3), (1, 1, 1), (130, 7, 40), (64, 33, 1)])
def test_diffusion_every_tile_ragged(marl, oracle_mod, dims):
    rng = np.random.default_rng(sum(dims))
    X, Y, Z = dims
    f0 = (rng.random((Z, Y, X, 12), dtype=np.float32) * np.float32(2.0)).astype(np.float32)
    occ = (rng.random((Z, Y, X)) < 0.15).astype(np.uint8)
    p = marl.default_params()
    cpu = f0.copy()
    oracle_mod.diffuse(cpu, occ, dims, p, 3)
    ctx = ctx_with(marl, dims, p, cells_at(marl, occ), f0, cap=max(int(occ.sum()), 1))
    lib = marl.load()
    tiles = 0
    while lib.marl_ctx_set_tile(ctx.h, tiles, 4) == 0:  # every tile shape the library offers
        tiles += 1
    assert tiles >= 12
    for tile in range(tiles):
        for zc in (1, 4, 13, 16):
            assert lib.marl_ctx_set_tile(ctx.h, tile, zc) == 0
            ctx.upload_field(f0)
            ctx.diffuse(3)
            np.testing.assert_array_equal(ctx.download_field(), cpu, err_msg=f"tile {tile} zc {zc}")


@pytest.mark.parametrize("mode", [0, 1])
def test_fused_sources(marl, oracle_mod, mode):
    dims = (40, 24, 20)
    rng = np.random.default_rng(4)
    f0 = (rng.random((20, 24, 40, 12), dtype=np.float32) * np.float32(9.8)).astype(np.float32)
    occ = (rng.random((20, 24, 40)) < 0.1).astype(np.uint8)
    p = marl.default_params()
    p.source_mode = mode
    ctx = ctx_with(marl, dims, p, cells_at(marl, occ), f0)
    ctx.diffuse(p.diffusion_substeps, fuse_sources=True)
    cpu = f0.copy()
    if mode == 0:
        oracle_mod.sources(cpu, dims, p)
    else:
        cpu[0, :, :, 1] = p.boundary_prime_oxidant
        cpu[0, :, :, 3] = p.boundary_prime_carbon
        cpu[-1, :, :, 2] = p.boundary_prime_reductant
    oracle_mod.diffuse(cpu, occ, dims, p, p.diffusion_substeps)
    np.testing.assert_array_equal(ctx.download_field(), cpu)
    # separate sources kernel + unfused diffusion gives the same result
    ctx.upload_field(f0)
    ctx.apply_boundary_sources()
    ctx.diffuse(p.diffusion_substeps)
    np.testing.assert_array_equal(ctx.download_field(), cpu)


def test_zero_substeps(marl, oracle_mod):
    dims = (16, 16, 8)
    f0 = wave_field(dims)
    p = marl.default_params()
    ctx = ctx_with(marl, dims, p, field=f0)
    ctx.diffuse(0, fuse_sources=True)  # sources only
    cpu = f0.copy()
    oracle_mod.sources(cpu, dims, p)
    np.testing.assert_array_equal(ctx.download_field(), cpu)


def test_seam_diffuse_tick_with_cells(marl, oracle_mod):
    """GpuFieldDiffuser::diffuse_tick_with_cells semantics (field_diffusion.rs:158-268)."""
    p = marl.default_params()
    f = wave_field(FULL)
    occ = occupancy_patterns(FULL)["dense_cluster"].astype(bool)
    cpu = f.copy()
    oracle_mod.diffuse(cpu, occ.astype(np.uint8), FULL, p, p.diffusion_substeps)
    ctx = marl.Context(FULL, p, cell_capacity=16)
    ctx.diffuse_tick_with_cells(f, occ)
    np.testing.assert_array_equal(f, cpu)
    # a second call continues from the caller's field
    oracle_mod.diffuse(cpu, occ.astype(np.uint8), FULL, p, p.diffusion_substeps)
    ctx.diffuse_tick_with_cells(f, occ)
    np.testing.assert_array_equal(f, cpu)
    # substeps == 0: Ok with no work
    p0 = p.copy()
    p0.diffusion_substeps = 0
    ctx0 = marl.Context(FULL, p0, cell_capacity=16)
    g = wave_field(FULL)
    ctx0.diffuse_tick_with_cells(g, occ)
    np.testing.assert_array_equal(g, wave_field(FULL))
    # size validation (InvalidInput)
    with pytest.raises(marl.MarlError) as e:
        ctx.diffuse_tick_with_cells(np.zeros(10, np.float32), occ)
    assert e.value.status_name == "INVALID_INPUT"
    with pytest.raises(marl.MarlError) as e:
        ctx.diffuse_tick_with_cells(f, occ[:, :, :5])
    assert e.value.status_name == "INVALID_INPUT"


@pytest.mark.parametrize("dims", [(128, 128, 64), (37, 19, 11)])
def test_diffuse_device_pointer_entry(marl, oracle_mod, dims):
    import torch

    X, Y, Z = dims
    rng = np.random.default_rng(8)
    f0 = rng.random((Z, Y, X, 12), dtype=np.float32)
    occ = (rng.random((Z, Y, X)) < 0.05).astype(np.uint8)
    p = marl.default_params()
    for substeps in (1, 4):
        field = torch.from_numpy(f0.copy()).cuda()
        scratch = torch.empty_like(field)
        o = torch.from_numpy(occ).cuda()
        stream = torch.cuda.current_stream().cuda_stream
        marl.diffuse_device(field.data_ptr(), scratch.data_ptr(), o.data_ptr(), dims, p, substeps, stream)
        cpu = f0.copy()
        oracle_mod.diffuse(cpu, occ, dims, p, substeps)
        np.testing.assert_array_equal(field.cpu().numpy(), cpu)


def light_case(marl, oracle_mod, dims, seed, absorber_hi=3.0, occ_frac=0.1):
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    f = (rng.random((Z, Y, X, 12), dtype=np.float32) * np.float32(absorber_hi)).astype(np.float32)
    occ = (rng.random((Z, Y, X)) < occ_frac).astype(np.uint8)
    p = marl.default_params()
    ctx = ctx_with(marl, dims, p, cells_at(marl, occ), f, cap=max(int(occ.sum()), 1))
    ctx.light_update()
    return ctx.download_light(), oracle_mod.light(f, occ, dims, p), oracle_mod.light_f64(f, occ, dims, p)


@pytest.mark.parametrize("dims", [(128, 128, 64), (33, 17, 70), (5, 3, 1)])
def test_light_matches_oracle(marl, oracle_mod, dims):
    gpu, cpu, cpu64 = light_case(marl, oracle_mod, dims, 3)
    np.testing.assert_allclose(gpu, cpu, rtol=LIGHT_RTOL, atol=LIGHT_ATOL)
    # exp differs from glibc expf by <= 1 ulp on a few voxels; a difference
    # then carries down the rest of its column
    assert np.mean(gpu == cpu) > 0.95
    # error against the FP64 oracle is no worse than the FP32 oracle's own
    err_gpu = np.abs(gpu - cpu64).max()
    err_cpu = np.abs(cpu - cpu64).max()
    assert err_gpu <= max(2 * err_cpu, 1e-6)


def test_light_floor_and_surface(marl, oracle_mod):
    gpu, cpu, _ = light_case(marl, oracle_mod, (8, 8, 64), 9, absorber_hi=400.0, occ_frac=0.3)
    assert (gpu[0] == 1.0).all()
    np.testing.assert_array_equal(gpu == 0, cpu == 0)  # the floor hits the same voxels
    np.testing.assert_allclose(gpu, cpu, rtol=LIGHT_RTOL, atol=LIGHT_ATOL)


def test_mass_f64(marl):
    rng = np.random.default_rng(12)
    dims = (64, 48, 40)
    f = rng.random((40, 48, 64, 12), dtype=np.float32)
    ctx = ctx_with(marl, dims, field=f)
    m = ctx.mass_f64()
    ref = f.reshape(-1, 12).astype(np.float64).sum(0)
    np.testing.assert_allclose(m, ref, rtol=1e-12)
    assert np.array_equal(m, ctx.mass_f64())  # fixed reduction order: reproducible
