"""CPU tests of the text input/output (csrc/textio.cpp): the parallel writer
against printf-style formatting done here in Python (correctly rounded, ties
to even on the exact binary value, as glibc's printf), and the parallel CRD
reader against the numbers it was written from."""
import numpy as np
import pytest


def _write(pac, path, balls, sol, E, T, Q):
    class R:
        edges, tris, tets = E, T, Q
    pac.write_complex(str(path), balls, sol, R)
    return path.read_bytes()


def _expected(balls, sol, E, T, Q):
    out = ["%d %d %d %d\n" % (len(balls), len(E), len(T), len(Q))]
    for x, y, z, r in balls:
        rr = np.float32(r) + np.float32(sol)
        out.append("%9.5f %9.5f %9.5f %9.5f\n" % (float(x), float(y), float(z), float(rr)))
    i32 = lambda a: a.astype(np.uint32).view(np.int32)
    out += ["%9d %9d\n" % tuple(e) for e in i32(E).tolist()]
    out += ["%9d %9d %9d\n" % tuple(t) for t in i32(T).tolist()]
    out += ["%9d %9d %9d %9d\n" % tuple(q) for q in i32(Q).tolist()]
    return "".join(out).encode()


def _awkward_floats(rng, n):
    """Values whose fixed-point form is hard to get right."""
    odd = rng.integers(0, 1 << 20, n) * 2 + 1
    v = [
        odd / 64.0,                      # x * 10^5 ends in exactly .5: ties
        -(odd / 64.0),
        odd / 128.0,
        rng.normal(0, 50, n),
        rng.normal(0, 1e-4, n),          # rounds to 0.00000 / -0.00000
        rng.uniform(-1e6, 1e6, n),
        10.0 ** rng.uniform(-40, 12, n) * rng.choice([-1, 1], n),
        np.full(n, 9.999995), np.full(n, 99999.999995), np.full(n, 0.000005),
    ]
    special = np.array([0.0, -0.0, 1e-45, -1e-45, 1.17e-38, 3.4e38, -3.4e38, 2.0 ** 40,
                        2.0 ** 40 - 2 ** 17, 123456789.0, 0.5e-5, 1.5e-5, 2.5e-5],
                       dtype=np.float64)
    return np.concatenate(v + [special]).astype(np.float32)


def test_writer_matches_printf_formatting(pac, tmp_path):
    rng = np.random.default_rng(5)
    f = _awkward_floats(rng, 400)
    m = len(f) // 4
    balls = f[: 4 * m].reshape(m, 4)
    sol = 1.4
    E = rng.integers(0, 1 << 32, (300, 2), dtype=np.uint64).astype(np.uint32)
    E[:10] = [[0, 1], [9, 10], [99999999, 100000000], [999999999, 1000000000],
              [2 ** 31 - 1, 2 ** 31], [2 ** 32 - 1, 5], [7, 123], [1, 2], [3, 4], [5, 6]]
    T = rng.integers(0, 3_000_000, (200, 3), dtype=np.uint64).astype(np.uint32)
    Q = rng.integers(0, 3_000_000, (100, 4), dtype=np.uint64).astype(np.uint32)
    got = _write(pac, tmp_path / "o.txt", balls, sol, E, T, Q)
    want = _expected(balls, sol, E, T, Q)
    if got != want:
        g, w = got.splitlines(), want.splitlines()
        bad = next(i for i in range(min(len(g), len(w))) if g[i] != w[i])
        pytest.fail("line %d: %r != %r" % (bad, g[bad], w[bad]))


def test_writer_many_blocks_in_order(pac, tmp_path):
    """More lines than one round of per-thread blocks: the blocks are
    written in order."""
    rng = np.random.default_rng(6)
    n_e = 2_300_000
    E = rng.integers(0, 10_000_000, (n_e, 2), dtype=np.uint64).astype(np.uint32)
    balls = rng.normal(0, 30, (70_000, 4)).astype(np.float32)
    e3 = np.zeros((0, 3), np.uint32)
    e4 = np.zeros((0, 4), np.uint32)
    got = _write(pac, tmp_path / "o.txt", balls, 0.0, E, e3, e4)
    want = _expected(balls, 0.0, E, e3, e4)
    assert got == want


def test_reader_large_file_any_whitespace(pac, tmp_path):
    rng = np.random.default_rng(7)
    n = 120_000  # a body of several MB: parsed in parallel
    balls = (rng.normal(0, 40, (n, 4)) * rng.choice([1, 1e-3, 1e3], (n, 4))).astype(np.float32)
    seps = [" ", "\t", "\n", "  \r\n", " \t "]
    parts = ["%d\n\n" % n]
    for i, b in enumerate(balls):
        for k in range(4):
            parts.append(repr(float(b[k])))
            parts.append(seps[(i + k) % len(seps)])
    parts.append("\n")
    p = tmp_path / "big.crd"
    p.write_text("".join(parts))
    got = pac.read_crd(str(p))
    assert got.tobytes() == balls.tobytes()


def test_reader_rejects_malformed_and_short(pac, tmp_path):
    p = tmp_path / "bad.crd"
    p.write_text("2\n1.0 2.0 3.0 1.5\n1.0 2.0x 3.0 1.5\n")
    with pytest.raises(pac.PacError) as ei:
        pac.read_crd(str(p))
    assert ei.value.status == -8
    p.write_text("2\n1.0 2.0 3.0 1.5\n1.0 2.0 3.0\n")
    with pytest.raises(pac.PacError):
        pac.read_crd(str(p))
    p.write_text("1\n1.0 2.0 3.0 1.5 7 8 9\n")  # extra numbers are ignored
    assert pac.read_crd(str(p)).tolist() == [[1.0, 2.0, 3.0, 1.5]]
