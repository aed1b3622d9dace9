"""The Python binding's copy of result lists out of the context's pinned
buffer (host only): results of 4 MB and more go in slices over the host's
threads, smaller ones are copied whole; every copy equals its source and
owns its memory."""
import numpy as np


def test_copy_many_equals_sources(pac):
    rng = np.random.default_rng(7)
    srcs = [rng.integers(0, 2**32, size=n, dtype=np.uint32)
            for n in (0, 1, 5, (16 << 20) // 4 - 1, (16 << 20) // 4, 9_000_001)]
    outs = pac._copy_many(srcs)
    assert len(outs) == len(srcs)
    for a, o in zip(srcs, outs):
        assert o.dtype == a.dtype and o.shape == a.shape
        assert np.array_equal(o, a)
        assert not np.shares_memory(o, a)


def test_copy_many_mid_size_result(pac):
    # three lists of a few MB together (a 100k-ball complex's shape, smaller)
    # are sliced over the threads
    rng = np.random.default_rng(11)
    srcs = [rng.integers(0, 2**32, size=n, dtype=np.uint32)
            for n in (400_001, 0, 700_003, 250_000)]
    for _ in range(2):  # the second call reuses the threads
        outs = pac._copy_many(srcs)
        assert [o.shape for o in outs] == [a.shape for a in srcs]
        for o, a in zip(outs, srcs):
            assert np.array_equal(o, a) and not np.shares_memory(o, a)


def test_views_reshape_like_the_lists(pac):
    # an empty list comes back as (0, k), a full one keeps its rows
    e = pac._copy_many([pac._view(None, 0, 2)])[0].reshape(-1, 2)
    assert e.shape == (0, 2)
    a = np.arange(12, dtype=np.uint32)
    t = pac._copy_many([a])[0].reshape(-1, 3)
    assert t.shape == (4, 3) and t[3, 2] == 11
