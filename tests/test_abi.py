"""The C-ABI library loads, exports every symbol include/marl_cuda.h declares,
and its plain-data layouts agree between C and Python.  No compute calls are
made here (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "marl_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(marl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(marl):
    lib = marl.load()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(marl.EXPORTED) <= set(names)


def test_struct_layouts_agree(oracle_mod, marl):
    lay = oracle_mod.struct_layout()
    assert lay[0] == ctypes.sizeof(marl.SimParams)
    assert lay[1] == marl.RULESET_DTYPE.itemsize
    assert lay[2] == marl.CELL_DTYPE.itemsize
    assert lay[3] == marl.CHANGE_DTYPE.itemsize
    assert lay[4] == marl.CELL_DTYPE.fields["lineage_id"][1]
    assert lay[5] == marl.CELL_DTYPE.fields["internal"][1]
    assert lay[6] == marl.CELL_DTYPE.fields["ruleset"][1]
    assert lay[7] == marl.RULESET_DTYPE.fields["reactions"][1]
    assert lay[8] == marl.RULESET_DTYPE.fields["effectors"][1]
    assert lay[9] == marl.RULESET_DTYPE.fields["fate"][1]


def test_default_params_identical_to_oracle(oracle_mod, marl):
    a = marl.default_params()
    b = oracle_mod.default_params()
    assert bytes(a) == bytes(b)


def test_canonical_ruleset_roundtrip(oracle_mod, marl):
    """536-byte payload of crates/marl-format/src/lib.rs:70-89."""
    c = oracle_mod.make_starter(1, [3, 4, 5], 99)
    payload = marl.pack_ruleset(c["ruleset"])
    assert len(payload) == 536
    # receptors 96 B, transport 8 x 10 B: first transporter = (0.7, 0.0, ext 1, int 1)
    assert np.frombuffer(payload[96:104], "<f4").tolist() == [np.float32(0.7), 0.0]
    assert payload[104:106] == bytes([1, 1])
    # reactions start at 176: reaction 0 = (2, 0, 5, 1, 0.15, 0.7, 0.1)
    assert payload[176:180] == bytes([2, 0, 5, 1])
    assert np.frombuffer(payload[180:192], "<f4").tolist() == pytest.approx([0.15, 0.7, 0.1])
    # trailing hgt_propensity, mutation_rate
    assert np.frombuffer(payload[528:536], "<f4").tolist() == pytest.approx([0.1, 0.05])
    back = marl.unpack_ruleset(payload)
    assert marl.pack_ruleset(back) == payload


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_no_device_fails_loudly(marl):
    with pytest.raises(marl.MarlError) as e:
        marl.Context((8, 8, 8))
    assert e.value.status_name in ("NO_DEVICE", "CUDA")


def test_invalid_dims_rejected_before_device(marl):
    lib = marl.load()
    h = ctypes.c_void_p()
    p = marl.default_params()
    st = lib.marl_ctx_create(0, 8, 8, ctypes.byref(p), 16, ctypes.byref(h))
    assert st == 1 and not h.value
    st = lib.marl_ctx_create(4096, 8, 8, ctypes.byref(p), 16, ctypes.byref(h))
    assert st == 1
