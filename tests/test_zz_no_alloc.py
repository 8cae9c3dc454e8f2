"""marl_diffuse_device_noalloc through the C ABI.

This entry point is for callers that cannot allocate device memory while they
run (their memory belongs to another allocator or a fixed pool, or an
allocation is not acceptable in their loop).  It must give exactly the result
of marl_diffuse_device, which allocates its scratch per call.  Two calls in a
row check that the shared static scratch array, which keeps the previous
call's contents, does not leak into the next result.  The file is named to be
collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_pair(marl, dims, substeps, seed):
    import torch

    X, Y, Z = dims
    rng = np.random.default_rng(seed)
    f0 = rng.random((Z, Y, X, 12), dtype=np.float32)
    occ = (rng.random((Z, Y, X)) < 0.08).astype(np.uint8)
    p = marl.default_params()
    stream = torch.cuda.current_stream().cuda_stream
    o = torch.from_numpy(occ).cuda()
    ref = torch.from_numpy(f0.copy()).cuda()
    scratch = torch.empty_like(ref)
    marl.diffuse_device(ref.data_ptr(), scratch.data_ptr(), o.data_ptr(), dims, p, substeps, stream)
    got = torch.from_numpy(f0.copy()).cuda()
    marl.diffuse_device_noalloc(got.data_ptr(), o.data_ptr(), dims, p, substeps, stream)
    return ref.cpu().numpy(), got.cpu().numpy()


@pytest.mark.parametrize("dims,substeps", [((64, 64, 64), 10), ((37, 21, 13), 3)])
def test_noalloc_matches_allocating_entry_twice(marl, dims, substeps):
    for call, seed in enumerate((1, 2)):  # two calls in a row, different inputs
        ref, got = run_pair(marl, dims, substeps, seed)
        np.testing.assert_array_equal(got, ref, err_msg=f"call {call}")  # bit-exact, as every diffusion test


def test_noalloc_rejects_oversized_grid(marl):
    import torch

    dims = (128, 128, 64)  # 1,048,576 voxels > 262,144
    f = torch.zeros((64, 128, 128, 12), dtype=torch.float32, device="cuda")
    o = torch.zeros((64, 128, 128), dtype=torch.uint8, device="cuda")
    with pytest.raises(marl.MarlError) as e:
        marl.diffuse_device_noalloc(f.data_ptr(), o.data_ptr(), dims, marl.default_params(), 1)
    assert e.value.status_name == "INVALID_INPUT"
