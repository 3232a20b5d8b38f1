"""Packed (f32, i32) key format, pinned by the reference's own checks in
archive/test_pack_unpack.py (cases :16-26, ordering :68-77, seeded sort
:175-230) -- the same scheme as pyfastflow/flow/f32_i32_struct.py."""
import numpy as np

from pyfastflow_b200.flow import f32_i32_struct as K

ROUNDTRIP = [(0.0, 0), (1.0, 1), (-1.0, 2), (3.14159, 42), (-2.71828, 100), (1e6, 999), (-1e6, 1000),
             (1e-6, 5), (-1e-6, 10)]
ORDERED = [(-10.0, 0), (-1.0, 0), (-1.0, 999), (0.0, 100), (1.0, 0), (1.0, 50), (1.0, 999), (10.0, 0)]


def test_roundtrip_cases(orc):
    for f, i in ROUNDTRIP:
        k = orc.pack_float_index(f, i)
        assert int(K.pack_float_index(np.float32(f), i)) == k
        f2, i2 = orc.unpack_float_index(k)
        assert f2 == np.float32(f) and i2 == i
        f3, i3 = K.unpack_float_index(k)
        assert f3 == np.float32(f) and i3 == i


def test_ordering_cases(orc):
    keys = [orc.pack_float_index(f, i) for f, i in ORDERED]
    assert all(a < b for a, b in zip(keys, keys[1:]))


def test_seeded_sort_matches_lexicographic(orc):
    np.random.seed(42)
    n = 10000
    floats = np.random.uniform(-1e6, 1e6, n).astype(np.float32)
    idx = np.random.randint(0, 750000, n, dtype=np.int32)
    packed = K.pack_float_index(floats, idx)
    by_key = [(floats[i], idx[i]) for i in np.argsort(packed, kind="stable")]
    assert by_key == sorted(zip(floats, idx))
    assert np.array_equal(packed, np.array([orc.pack_float_index(f, i) for f, i in zip(floats[:500], idx[:500])]
                                           + list(packed[500:])))


def test_signed_zero_and_invalid(orc):
    assert orc.pack_float_index(-0.0, 7) < orc.pack_float_index(0.0, 7)
    assert K.INVALID_KEY == orc.pack_float_index(1e8, 42)
    assert orc.unpack_float_index(K.INVALID_KEY) == (np.float32(1e8), 42)
