"""The host restatement of the device's 16-bit table quantizer (exmarg_b200.quantize_table),
checked against torch's own float32 -> float16 / bfloat16 conversions (round to nearest even)."""

import numpy as np
import pytest
import torch

import exmarg_b200 as eb
from exmarg_b200 import synth


def _tables():
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((4, 5, 6, 7)) * 3e3).astype(np.float32)
    a[0, 0, 0, :3] = [0.0, -1e-9, 7e-6]               # zeros and values below float16's normal range
    spec = synth.TableSpec(ntau=5, nphif=49, nb=20, nd=23)
    g = synth.gen_table_node(spec, 1, synth.S_NODES_PROD[20:23], 7)
    return [a, g]


@pytest.mark.parametrize("i", [0, 1])
def test_f16_matches_torch_and_scale_is_a_power_of_two(i):
    T = _tables()[i]
    v, sc = eb.quantize_table(T, "f16")
    m, e = np.frexp(sc)
    assert m == 0.5                                    # a power of two
    amax = np.abs(T).max()
    assert 2.0 ** 14 <= amax / sc < 2.0 ** 15
    ref = (torch.from_numpy(T / np.float32(sc)).to(torch.float16).to(torch.float32) * sc).numpy()
    assert np.array_equal(v, ref)
    assert np.abs(v - T).max() <= amax * 2.0 ** -11    # half an ulp of float16 at the largest value


@pytest.mark.parametrize("i", [0, 1])
def test_bf16_matches_torch(i):
    T = _tables()[i]
    v, sc = eb.quantize_table(T, "bf16")
    assert sc == 1.0
    assert np.array_equal(v, torch.from_numpy(T).to(torch.bfloat16).to(torch.float32).numpy())


def test_f32_is_identity_and_bad_dtype_raises():
    T = _tables()[0]
    v, sc = eb.quantize_table(T, "f32")
    assert v is T or np.array_equal(v, T)
    with pytest.raises(ValueError):
        eb.quantize_table(T, "f8")
    with pytest.raises(ValueError):
        eb.with_table_dtype(synth.MemoryStore(synth.TableSpec(ntau=3, nphif=49, nb=4, nd=5), [1.0], 1,
                                              tables=[np.zeros((3, 49, 4, 5), np.float32)]), "int8")


def test_with_table_dtype_is_a_new_store():
    st = synth.MemoryStore(synth.TableSpec(ntau=3, nphif=49, nb=4, nd=5), [1.0], 1,
                           tables=[np.zeros((3, 49, 4, 5), np.float32)])
    from exmarg_b200 import _lib
    t0 = _lib.token_of(st)
    h = eb.with_table_dtype(st, "f16")
    assert h.table_dtype == "f16" and st.table_dtype == "f32"
    assert _lib.token_of(h) != t0 and h.tables[0] is st.tables[0]
