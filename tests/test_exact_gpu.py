"""GPU tests of the decision-exact predicate mode (PAC_PRED_EXACT): the
engine's FP64 filter + 640-bit integer cascade against the restatement's
exact mode (extended-precision filter + arbitrary-precision integers,
itself pinned to rational arithmetic in test_exact_oracle.py)."""
import numpy as np
import pytest

from conftest import canonical, golden

pytestmark = pytest.mark.gpu


def _exact(pac, **kw):
    return pac.Engine(device=0, predicates="exact", **kw)


def _same(res, E, T, Q):
    np.testing.assert_array_equal(res.edges, E)
    np.testing.assert_array_equal(res.tris, T)
    np.testing.assert_array_equal(res.tets, Q)


@pytest.mark.parametrize("case", ["globule", "snapped", "lattice", "1grm"])
def test_exact_mode_matches_exact_oracle(pac, orc, case):
    if case == "globule":
        balls, sol, alpha = pac.globule(2500, seed=pac.SEED_BASE + 61), 1.4, 1.0
    elif case == "snapped":
        balls, sol, alpha = pac.snapped_globule(2500, seed=pac.SEED_BASE + 62), 1.4, 1.0
    elif case == "lattice":
        g = np.stack(np.meshgrid(np.arange(6), np.arange(6), np.arange(4), indexing="ij"), -1)
        balls = np.concatenate([g.reshape(-1, 3), np.full((g.size // 3, 1), 1.5)], 1)
        balls, sol, alpha = balls.astype(np.float32), 0.0, 0.5
    else:
        balls, sol, alpha = golden("1grm_ld_alpha1")[0], 0.0, 1.0
    e, t, q, st = orc.alpha_complex(balls, sol, alpha, exact=True)
    with _exact(pac) as eng:
        r = eng.alpha_complex(balls, sol, alpha)
    _same(r, e, t, q)
    for k in ("cand_edges", "alpha_edges", "cand_tris", "alpha_tris", "cand_tets", "alpha_tets"):
        assert r.stats[k] == st[k], k
    assert r.stats["filter_evals"] > r.stats["cand_edges"]
    print("%s: %d filtered decisions, %d integer fallbacks (%.2e), %d SoS"
          % (case, r.stats["filter_evals"], r.stats["exact_fallbacks"],
             r.stats["exact_fallbacks"] / r.stats["filter_evals"], r.stats["sos_calls"]))
    if case in ("snapped", "lattice"):
        assert r.stats["exact_fallbacks"] > 0


def test_exact_mode_differs_from_reference_arithmetic_only_on_ties(pac):
    """On the lattice-snapped globule the reference's single-precision tests
    flip some ties; everywhere else the two modes agree."""
    balls = pac.snapped_globule(2500, seed=pac.SEED_BASE + 62)
    with _exact(pac) as eng:
        x = eng.alpha_complex(balls, 1.4, 1.0)
    with pac.Engine(device=0) as eng:
        f = eng.alpha_complex(balls, 1.4, 1.0)
    d = [len(set(map(tuple, canonical(a))) ^ set(map(tuple, canonical(b))))
         for a, b in ((x.edges, f.edges), (x.tris, f.tris), (x.tets, f.tets))]
    total = len(x.edges) + len(x.tris) + len(x.tets)
    assert 0 < sum(d) < 0.01 * total


def test_exact_mode_as_run_and_batched(pac, orc):
    balls = pac.snapped_globule(1200, seed=pac.SEED_BASE + 63)
    e, t, q, _ = orc.alpha_complex(balls, 1.4, 1.0, tet_ortho=False, exact=True)
    with _exact(pac, tet_mode="as-run") as eng:
        _same(eng.alpha_complex(balls, 1.4, 1.0), e, t, q)
    sizes = np.array([300, 1200, 700])
    mols = [pac.snapped_globule(int(m), seed=pac.SEED_BASE + 70 + k) for k, m in enumerate(sizes)]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    with _exact(pac) as eng:
        res, _ = eng.alpha_complex_batch(np.concatenate(mols), off, 1.4, 0.5)
    for m, b in enumerate(mols):
        e, t, q, _ = orc.alpha_complex(b, 1.4, 0.5, exact=True)
        _same(res[m], e, t, q)
