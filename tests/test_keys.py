"""Packed (f32, i32) key format, pinned by the reference's own checks in
archive/test_pack_unpack.py (cases :16-26, ordering :68-77, seeded sort
:175-230) -- the same scheme as pyfastflow/flow/f32_i32_struct.py -- and by the
atomic lexicographic argmin experiment archive/expe_lexicographic_argmin/t1.py
:63-175 (an atomic min over packed keys is the (value, then index) argmin)."""
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


def test_atomic_min_is_lexicographic_argmin(orc):
    """t1.py:63-175: 100 values uniform in [-100, 100) with indices 0..99, the value at
    position 56 replaced by -99.5 with index 999; min over the packed keys must be
    the manual lexicographic scan's (value, then index) winner.  Ties added at
    both a larger and a smaller index check the index tie-break, which the saddle
    pass's atomicMin (lakeflow.py:164-194) relies on."""
    rng = np.random.default_rng(63)
    vals = (rng.random(100) * 200.0 - 100.0).astype(np.float32)
    idx = np.arange(100, dtype=np.int32)
    vals[56], idx[56] = np.float32(-99.5), 999

    def manual(v, ix):  # t1.py's verification loop
        mv, mi = v[0], ix[0]
        for a, b in zip(v[1:], ix[1:]):
            if a < mv or (a == mv and b < mi):
                mv, mi = a, b
        return mv, mi

    for extra in ([], [(np.float32(-99.5), 1200)], [(np.float32(-99.5), 7)], [(np.float32(-100.0), 3)]):
        v = np.concatenate([vals, np.array([e[0] for e in extra], np.float32)])
        ix = np.concatenate([idx, np.array([e[1] for e in extra], np.int32)])
        keys = K.pack_float_index(v, ix)
        got = K.unpack_float_index(int(keys.min()))
        assert (np.float32(got[0]), int(got[1])) == manual(v, ix)
        assert int(keys.min()) == min(orc.pack_float_index(a, int(b)) for a, b in zip(v, ix))
