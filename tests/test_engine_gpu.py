"""GPU parity tests: the CUDA engine, called through the C ABI, against the
reference's shipped outputs and against the CPU restatement, bit for bit
and in the reference binary's output order."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, canonical, golden

pytestmark = pytest.mark.gpu

FORMULA = {0: "upstream", 1: "plain-xmp"}


def _engine(pac, formula=0, tet_mode="as-written", predicates="strict"):
    return pac.Engine(device=0, formula=FORMULA[formula], tet_mode=tet_mode, predicates=predicates)


def _same(res, E, T, Q):
    np.testing.assert_array_equal(res.edges, E)
    np.testing.assert_array_equal(res.tris, T)
    np.testing.assert_array_equal(res.tets, Q)


# ------------------------------------------------------------ shipped outputs
@pytest.mark.parametrize("name,formula", [("1grm_ld_alpha1", 0), ("1grm_plain_alpha1", 1)])
def test_golden_outputs_as_run(pac, name, formula):
    balls, E, T, Q = golden(name)
    with _engine(pac, formula, "as-run") as eng:
        _same(eng.alpha_complex(balls, 0.0, 1.0), E, T, Q)


def test_golden_1k4c_against_restatement(pac, orc):
    balls, E, T, Q = golden("1k4c_plain_alpha1")
    for mode, flag in (("as-run", False), ("as-written", True)):
        e, t, q, _ = orc.alpha_complex(balls, 0.0, 1.0, orc.PLAIN_XMP, tet_ortho=flag)
        with _engine(pac, 1, mode) as eng:
            _same(eng.alpha_complex(balls, 0.0, 1.0), e, t, q)


# ------------------------------------------------------------ synthetic cases
CASES = [
    # n, seed offset, sol, alpha, snapped
    (300, 0, 0.0, 0.0, False),
    (1300, 0, 0.0, 0.0, False),      # the 1,300-ball plain case
    (1300, 0, 1.4, 1.0, False),
    (2000, 1, 1.4, 1.0, True),       # lattice-snapped: exact zeros, SoS
    (3000, 7, 1.4, 0.5, False),
    (800, 9, 0.5, 2.0, True),
]


@pytest.mark.parametrize("n,seed,sol,alpha,snap", CASES)
@pytest.mark.parametrize("formula", [0, 1])
def test_synthetic_against_restatement(pac, orc, n, seed, sol, alpha, snap, formula):
    balls = (pac.snapped_globule(n, seed=pac.SEED_BASE + seed) if snap
             else pac.globule(n, seed=pac.SEED_BASE + seed))
    for mode, flag in (("as-written", True), ("as-run", False)):
        if mode == "as-run" and n > 2000 and sol > 0:
            continue  # as-run output grows ~2700 tetrahedra per ball
        e, t, q, st = orc.alpha_complex(balls, sol, alpha, formula, tet_ortho=flag)
        with _engine(pac, formula, mode) as eng:
            r = eng.alpha_complex(balls, sol, alpha)
        _same(r, e, t, q)
        for k in ("cand_edges", "alpha_edges", "cand_tris", "alpha_tris", "cand_tets",
                  "alpha_tets"):
            assert r.stats[k] == st[k], k
        if flag:
            # the engine defers exact zeros and evaluates SoS only for a
            # tetrahedron that no other ball already rejects
            assert r.stats["sos_calls"] <= st["sos_calls"]


@pytest.mark.slow
def test_degenerate_25k_as_written(pac, orc):
    """The 25,000-ball lattice-snapped stress case (sol 1.4, alpha 1)."""
    balls = pac.snapped_globule(25000, seed=pac.SEED_BASE + 1)
    e, t, q, st = orc.alpha_complex(balls, 1.4, 1.0, orc.UPSTREAM, tet_ortho=True)
    with _engine(pac, 0, "as-written") as eng:
        r = eng.alpha_complex(balls, 1.4, 1.0)
    _same(r, e, t, q)
    assert st["sos_calls"] > 0 and r.stats["sos_calls"] <= st["sos_calls"]


# ------------------------------------------------------------ edge cases
@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 5])
def test_tiny_inputs(pac, orc, n):
    balls = np.array([[0, 0, 0, 1.7], [1.5, 0, 0, 1.6], [0.4, 1.3, 0, 1.5],
                      [0.5, 0.5, 1.2, 1.8], [1.1, 1.0, 1.1, 1.52]], np.float32)[:n]
    for mode, flag in (("as-written", True), ("as-run", False)):
        with _engine(pac, 0, mode) as eng:
            r = eng.alpha_complex(balls, 1.4, 1.0)
        if n == 0:
            assert r.counts() == (0, 0, 0)
            continue
        e, t, q, _ = orc.alpha_complex(balls, 1.4, 1.0, 0, tet_ortho=flag)
        _same(r, e, t, q)


def test_coplanar_and_cospherical_lattice(pac, orc):
    """All centres on a 1 A cubic lattice with equal radii: every insphere
    test is degenerate somewhere, SoS decides."""
    g = np.stack(np.meshgrid(np.arange(6), np.arange(6), np.arange(4), indexing="ij"), -1)
    balls = np.concatenate([g.reshape(-1, 3), np.full((g.size // 3, 1), 1.5)], 1).astype(np.float32)
    for formula in (0, 1):
        e, t, q, st = orc.alpha_complex(balls, 0.0, 0.5, formula, tet_ortho=True)
        with _engine(pac, formula, "as-written") as eng:
            r = eng.alpha_complex(balls, 0.0, 0.5)
        _same(r, e, t, q)
        assert st["sos_calls"] > 0


def test_far_apart_and_duplicate_free_sparse(pac, orc):
    rng = np.random.default_rng(3)
    balls = np.concatenate([rng.uniform(-300, 300, (200, 3)), np.full((200, 1), 1.7)], 1)
    balls = balls.astype(np.float32)
    e, t, q, _ = orc.alpha_complex(balls, 1.4, 1.0, 0, tet_ortho=True)
    with _engine(pac, 0) as eng:
        _same(eng.alpha_complex(balls, 1.4, 1.0), e, t, q)


def test_non_finite_input_rejected(pac):
    balls = np.array([[0, 0, 0, 1.7], [np.nan, 0, 0, 1.6]], np.float32)
    with _engine(pac) as eng:
        with pytest.raises(pac.PacError) as ei:
            eng.alpha_complex(balls, 1.4, 1.0)
        assert ei.value.status == -1
        # the context stays usable
        r = eng.alpha_complex(balls[:1], 1.4, 1.0)
        assert r.counts() == (0, 0, 0)


def test_degree_limit_reported(pac):
    """A clump denser than any molecule exceeds the supported upper degree:
    a clear capacity error, and the context stays usable."""
    rng = np.random.default_rng(1)
    balls = np.concatenate([rng.uniform(0, 4, (600, 3)), np.full((600, 1), 1.7)], 1)
    with _engine(pac) as eng:
        with pytest.raises(pac.PacError) as ei:
            eng.alpha_complex(balls.astype(np.float32), 1.4, 1.0)
        assert ei.value.status == -3
        r = eng.alpha_complex(pac.globule(300), 1.4, 1.0)
        assert r.counts()[0] > 0


def test_deterministic_reruns(pac):
    balls = pac.globule(5000, seed=99)
    with _engine(pac) as eng:
        a = eng.alpha_complex(balls, 1.4, 1.0)
        b = eng.alpha_complex(balls, 1.4, 1.0)
    _same(a, b.edges, b.tris, b.tets)


# ------------------------------------------------------------ batched mode
def test_batch_equals_per_molecule(pac):
    sizes = np.array([250, 1, 0, 700, 1200, 3, 400], np.uint32)
    balls, off = pac.batch(sizes, seed=77)
    with _engine(pac) as eng:
        res, st = eng.alpha_complex_batch(balls, off, 1.4, 0.5)
        assert len(res) == len(sizes)
        for m in range(len(sizes)):
            single = eng.alpha_complex(balls[off[m]:off[m + 1]], 1.4, 0.5)
            _same(res[m], single.edges, single.tris, single.tets)


# ------------------------------------------------------------ device API
class _DeviceView:
    """__cuda_array_interface__ over a raw device pointer (uint32)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4",
                                         "data": (ptr, False), "version": 2}


def _device_list(ptr, rows, k):
    import ctypes
    import torch
    if rows == 0:
        return np.zeros((0, k), np.uint32)
    addr = ctypes.cast(ptr, ctypes.c_void_p).value
    t = torch.as_tensor(_DeviceView(addr, rows * k), device="cuda")
    return t.cpu().numpy().view(np.uint32).reshape(rows, k)


def test_device_entry_point(pac):
    import torch
    balls = pac.globule(2000, seed=4)
    with _engine(pac) as eng:
        host = eng.alpha_complex(balls, 1.4, 1.0)
        d = torch.from_numpy(balls).cuda()
        torch.cuda.synchronize()
        cx, st = eng.alpha_complex_device(d.data_ptr(), len(balls), 1.4, 1.0)
        assert cx.on_device == 1 and st["kernels_launched"] > 0
        np.testing.assert_array_equal(_device_list(cx.edges, cx.n_edges, 2), host.edges)
        np.testing.assert_array_equal(_device_list(cx.tris, cx.n_tris, 3), host.tris)
        np.testing.assert_array_equal(_device_list(cx.tets, cx.n_tets, 4), host.tets)


# ------------------------------------------------------------ CLI
def test_cli_report_phases_and_progress(pac, tmp_path):
    """The CLI's report follows the reference's: one "Processed N atoms"
    line per reference chunk (512 doubled up to the suggestion,
    AlphaComplexLargeData.cu:1227-1235) and, as written, the
    empty-orthosphere test reported as its own phase ("AC2 test for
    tetrahedra", AlphaComplexLargeData.cu:2014)."""
    balls = pac.globule(3000, seed=pac.SEED_BASE + 5)
    crd = tmp_path / "g.crd"
    with open(crd, "w") as f:
        f.write("%d\n" % len(balls))
        for b in balls:
            f.write("%s %s %s %s\n" % tuple(repr(float(v)) for v in b))
    exe = os.path.join(pac.BIN_DIR, "parallelac-largeData")
    r = subprocess.run([exe, str(crd), str(tmp_path / "o.txt"), "1.4", "1", "1000"],
                       capture_output=True, text=True,
                       env=dict(os.environ, PAC_TET_MODE="as-written"))
    assert r.returncode == 0, r.stderr
    starts = [int(l.split()[1]) for l in r.stdout.splitlines() if l.startswith("Processed")]
    assert starts == [0, 1024, 2048]
    ac2 = [l for l in r.stdout.splitlines() if l.startswith("AC2 test for tetrahedra:")]
    assert len(ac2) == 1 and float(ac2[0].split(":")[1]) > 0.0


def test_cli_reproduces_golden_file(pac, tmp_path):
    import gzip
    balls, _, _, _ = golden("1grm_ld_alpha1")
    crd = tmp_path / "1grm.crd"
    with open(crd, "w") as f:
        f.write("%d\n" % len(balls))
        for b in balls:
            f.write("%s %s %s %s\n" % tuple(repr(float(v)) for v in b))
    out = tmp_path / "out.txt"
    exe = os.path.join(pac.BIN_DIR, "parallelac-largeData")
    r = subprocess.run([exe, str(crd), str(out), "0", "1", "100000"], capture_output=True,
                       text=True, env=dict(os.environ, PAC_TET_MODE="as-run"))
    assert r.returncode == 0, r.stderr
    assert "Number of tetrahedra:           183" in r.stdout
    assert out.read_bytes() == gzip.open(os.path.join(GOLDEN, "1grm_ld_alpha1.txt.gz")).read()
    r = subprocess.run([exe, str(crd)], capture_output=True, text=True)
    assert r.returncode == 1 and r.stdout.startswith("Usage : parallelac-largeData")


# ------------------------------------------------------------ FMA flavour
def test_fma_flavour_runs_and_is_close(pac, orc):
    """The contraction-enabled flavour follows the reference binary's default
    build; against the strict flavour it may differ only on near ties."""
    balls = pac.globule(3000, seed=21)
    with _engine(pac, 0, "as-written", "strict") as a, _engine(pac, 0, "as-written", "fma") as b:
        ra, rb = a.alpha_complex(balls, 1.4, 1.0), b.alpha_complex(balls, 1.4, 1.0)
    for x, y in ((ra.edges, rb.edges), (ra.tris, rb.tris), (ra.tets, rb.tets)):
        sx, sy = set(map(tuple, canonical(x))), set(map(tuple, canonical(y)))
        assert len(sx ^ sy) <= max(5, len(sx) // 1000)


# ------------------------------------------------------------ reference runs
def _refrun(name, build):
    d = np.load(os.path.join(GOLDEN, "refrun", "refrun_%s__%s.npz" % (name, build)))
    return d["edges"], d["tris"], d["tets"]


def test_engine_matches_reference_binary_nofma(pac):
    """Strict flavour == the reference built with -fmad=false (rr128), in order."""
    cases = {"1grm_a1": (golden("1grm_ld_alpha1")[0], 0.0, 1.0),
             "1k4c_a1": (golden("1k4c_plain_alpha1")[0], 0.0, 1.0),
             "glob1300_a0": (pac.globule(1300, seed=pac.SEED_BASE), 0.0, 0.0)}
    with _engine(pac, 0, "as-written", "strict") as eng:
        for name, (balls, sol, alpha) in cases.items():
            _same(eng.alpha_complex(balls, sol, alpha), *_refrun(name, "rr128-nofma"))


def test_engine_matches_reference_digest_5000(pac):
    import hashlib
    import json
    man = json.load(open(os.path.join(GOLDEN, "refrun", "refrun_manifest.json")))
    balls = pac.globule(5000, seed=pac.SEED_BASE + 4)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()
    with _engine(pac, 0, "as-written", "strict") as eng:
        r = eng.alpha_complex(balls, 1.4, 1.0)
    assert [sha(r.edges), sha(r.tris), sha(r.tets)] == \
        man["glob5000_s14_a1"]["builds"]["rr128-nofma"]["sha256"]


def test_fma_flavour_against_reference_default_contraction(pac):
    """The contraction flavour against the reference built with nvcc's
    default -fmad=true (rr128) on 1k4c.  Which multiply-adds nvcc fuses
    depends on the code around each expression, so no build of different
    kernels can match that binary bit for bit; the flavour is the closer
    approximation: fewer differing simplices than the strict flavour
    (which differs from that build in 82 of ~118k)."""
    balls = golden("1k4c_plain_alpha1")[0]
    E, T, Q = _refrun("1k4c_a1", "rr128")

    def diff(pred):
        with _engine(pac, 0, "as-written", pred) as eng:
            r = eng.alpha_complex(balls, 0.0, 1.0)
        return [len(set(map(tuple, canonical(a))) ^ set(map(tuple, canonical(b))))
                for a, b in ((r.edges, E), (r.tris, T), (r.tets, Q))]
    fma, strict = diff("fma"), diff("strict")
    print("vs the reference's default-contraction build, differing (edges, tris, tets): "
          "fma flavour %s, strict flavour %s" % (fma, strict))
    assert sum(strict) == 82
    assert sum(fma) < sum(strict)


def test_chunked_tetrahedron_queue(pac, orc):
    """A queue far smaller than the alpha tetrahedra of the pass: the balls
    are processed in many chunks (with overflow retries); same lists."""
    balls = pac.globule(4000, seed=pac.SEED_BASE + 12)
    e, t, q, st = orc.alpha_complex(balls, 1.4, 1.0, orc.UPSTREAM, tet_ortho=True)
    with pac.Engine(tet_mode="as-written", queue_entries=200_000) as eng:
        r = eng.alpha_complex(balls, 1.4, 1.0)
    _same(r, e, t, q)
    assert r.stats["alpha_tets"] == st["alpha_tets"] and r.stats["cand_tets"] == st["cand_tets"]


def test_verbose_reports_chunks_and_stages(pac, capfd):
    """verbose: one line per tetrahedron chunk (its counts add up to the
    pass's) and one line of stage timings per pass, on stderr."""
    balls = pac.globule(4000, seed=pac.SEED_BASE + 12)
    with pac.Engine(tet_mode="as-written", queue_entries=200_000, verbose=True) as eng:
        r = eng.alpha_complex(balls, 1.4, 1.0)
    err = capfd.readouterr().err
    chunks = [l for l in err.splitlines() if l.startswith("[pac] tetrahedra of balls")]
    assert len(chunks) > 1
    alpha = sum(int(l.split(": ")[1].split(", ")[1].split()[0]) for l in chunks)
    assert alpha == r.stats["alpha_tets"]
    assert any(l.startswith("[pac] %d balls: grid" % len(balls)) for l in err.splitlines())


@pytest.mark.slow
def test_assembly_2p5m_matches_restatement_digest(pac):
    """The large single pass: 2.5M balls (400 globules of 6,250
    in an 8 x 10 x 5 grid at 60 A pitch), sol 1.4, alpha 1, as written, in
    one call (the tetrahedron queue runs in chunks); lists and stage counts
    against the restatement's digests (tests/golden/make_assembly_digest.py)."""
    import hashlib
    import json
    man = json.load(open(os.path.join(GOLDEN, "assembly_2p5m.json")))
    balls = pac.assembly()
    assert hashlib.sha256(balls.tobytes()).hexdigest() == man["input_sha256"]

    def sha(a):
        return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()
    rec = man["as-written"]
    with _engine(pac, 0, "as-written") as eng:
        r = eng.alpha_complex(balls, 1.4, 1.0)
    assert [len(r.edges), len(r.tris), len(r.tets)] == rec["counts"]
    assert [sha(r.edges), sha(r.tris), sha(r.tets)] == rec["sha256"]
    for k in ("cand_edges", "alpha_edges", "cand_tris", "alpha_tris", "cand_tets", "alpha_tets"):
        assert r.stats[k] == rec["stats"][k], k
    print("2.5M assembly: %.1f ms, %d simplices" % (r.stats["ms_total"], sum(rec["counts"])))


def test_autotuner_passes_all_give_the_same_lists(pac, orc):
    """With autotune on, the first passes of a context each run another
    launch shape; every pass, tuning or tuned, returns the same lists."""
    balls = pac.globule(3000, seed=pac.SEED_BASE + 81)
    e, t, q, _ = orc.alpha_complex(balls, 1.4, 1.0, orc.UPSTREAM, tet_ortho=True)
    with pac.Engine(autotune=True) as eng:
        for _ in range(14):  # 12 candidate shapes, then the chosen one
            _same(eng.alpha_complex(balls, 1.4, 1.0), e, t, q)
    with pac.Engine(enum_blocks=2, scan_blocks=2, heavy_blocks=3, unit_rows=3, scan_claim=64) as eng:
        _same(eng.alpha_complex(balls, 1.4, 1.0), e, t, q)


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


@pytest.mark.parametrize("refute", [True, False])
def test_headline_100k_matches_restatement_digest(pac, refute):
    """The workload the bench's headline is quoted on: the 100,000-ball
    globule plus 8 corner balls, sol 1.4, alpha 1, upstream formulas, as
    written, strict -- lists in reference order and the six stage counters
    against the restatement's digests (tests/golden/make_headline_digest.py),
    with and without the enumeration's early refutation."""
    import hashlib
    import json
    man = json.load(open(os.path.join(GOLDEN, "headline_100k.json")))
    balls = pac.pad_corners(pac.globule(100_000, seed=pac.SEED_BASE + 4))
    assert hashlib.sha256(balls.tobytes()).hexdigest() == man["input_sha256"]
    with pac.Engine(tet_mode="as-written", refute=refute) as eng:
        r = eng.alpha_complex(balls, 1.4, 1.0)
    assert [len(r.edges), len(r.tris), len(r.tets)] == man["counts"]
    assert [_sha(r.edges), _sha(r.tris), _sha(r.tets)] == man["sha256"]
    for k, v in man["stats"].items():
        assert r.stats[k] == v, k
    if refute:
        # most alpha tetrahedra never reach the queue
        assert r.stats["early_refuted"] > 0.5 * r.stats["alpha_tets"]
    else:
        assert r.stats["early_refuted"] == 0


def test_certified_filter_agrees_with_replay_on_gpu(pac):
    """Verify mode: the scan replays the reference's binary32 insphere for
    every decision the certified filter takes and counts disagreements --
    on a generic globule and on lattice-snapped inputs (exact ties)."""
    for balls in (pac.globule(20_000, seed=pac.SEED_BASE + 4),
                  pac.snapped_globule(5_000, seed=pac.SEED_BASE + 1)):
        with pac.Engine(tet_mode="as-written", verify=True, refute=False) as eng:
            r = eng.alpha_complex(balls, 1.4, 1.0)
        st = r.stats
        print("certified %d of %d insphere decisions, %d disagreements"
              % (st["cert_decisions"], st["insphere_evals"], st["cert_disagreements"]))
        assert st["cert_disagreements"] == 0
        assert st["cert_decisions"] > 0.9 * st["insphere_evals"]


@pytest.mark.slow
def test_batch_4096_matches_restatement_digests(pac):
    """The batched configuration in full: 4,096 molecules of log-uniform
    size in [200, 20000] (17.47 M balls), sol 1.4, alpha 0.5, as written, in
    one pac_alpha_complex_batch call; every molecule's lists against the
    restatement's (tests/golden/batch_4096.json: per-molecule list lengths
    and a sha256 per list kind over all molecules in order)."""
    import hashlib
    import json
    man = json.load(open(os.path.join(GOLDEN, "batch_4096.json")))
    sizes = pac.batch_sizes(4096)
    balls, off = pac.batch(sizes)
    assert hashlib.sha256(balls.tobytes()).hexdigest() == man["input_sha256"]
    with pac.Engine(tet_mode="as-written") as eng:
        res, st = eng.alpha_complex_batch(balls, off, 1.4, 0.5)
    got = np.array([r.counts() for r in res], dtype=np.int64)
    want = np.stack([man["edges_per_molecule"], man["tris_per_molecule"],
                     man["tets_per_molecule"]], 1)
    bad = np.nonzero((got != want).any(1))[0]
    assert len(bad) == 0, "molecules with other list lengths: %s" % bad[:10]
    h = [hashlib.sha256() for _ in range(3)]
    for r in res:
        for k, a in enumerate((r.edges, r.tris, r.tets)):
            h[k].update(np.ascontiguousarray(a, dtype=np.uint32).tobytes())
    assert [x.hexdigest() for x in h] == man["sha256_concat"]
    print("batch of 4,096: %d simplices, %.0f ms" % (got.sum(), st["ms_total"]))


@pytest.mark.parametrize("name", ["plain_1grm_a1", "plain_1k4c_a1", "plain_glob1300_a0",
                                  "plain_glob5000_s14_a1", "plain_glob3000_s14_a05"])
def test_engine_matches_plain_reference_binary(pac, name):
    """Plain-xmp formulas (AlphaComplexParallel.cu:203-230, 310-372), as
    written, strict flavour == the reference's plain binary built with
    -maxrregcount=128 -fmad=false and run on a B200, list for list in the
    binary's output order (fixtures by tests/golden/make_refrun_golden.py)."""
    import json
    man = json.load(open(os.path.join(GOLDEN, "refrun", "refrun_manifest.json")))[name]
    src = {"plain_1grm_a1": lambda: golden("1grm_ld_alpha1")[0],
           "plain_1k4c_a1": lambda: golden("1k4c_plain_alpha1")[0],
           "plain_glob1300_a0": lambda: pac.globule(1300, seed=pac.SEED_BASE),
           "plain_glob5000_s14_a1": lambda: pac.pad_corners(pac.globule(5000, seed=pac.SEED_BASE + 4)),
           "plain_glob3000_s14_a05": lambda: pac.pad_corners(pac.globule(3000, seed=pac.SEED_BASE + 7))}
    balls = src[name]()
    assert len(balls) == man["n"]
    with _engine(pac, 1, "as-written", "strict") as eng:
        r = eng.alpha_complex(balls, man["sol_rad"], man["alpha"])
    _same(r, *_refrun(name, "plain-rr128-nofma"))



@pytest.mark.parametrize("world", [2, 3])
def test_slab_passes_partition_the_complex(pac, orc, world):
    """The engine's slab passes (Engine(slab=(r, world)), one after the other
    on this GPU): each equals the restatement's simplices owned by the slab
    (pac.slab_cuts, the ownership rule the multi-rank gather relies on), and
    together in rank order they are the single pass's lists."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_multirank import slab_expectation
    balls = pac.assembly(nx=2, ny=2, nz=2, per=2500)
    full, shares = slab_expectation(pac, orc, balls, 1.4, 1.0, world)
    with _engine(pac) as eng:
        one = eng.alpha_complex(balls, 1.4, 1.0)
    _same(one, *full)
    cat = [[], [], []]
    for r in range(world):
        with pac.Engine(tet_mode="as-written", slab=(r, world)) as eng:
            part = eng.alpha_complex(balls, 1.4, 1.0)
        _same(part, *shares[r])
        for k, a in enumerate((part.edges, part.tris, part.tets)):
            cat[k].append(a)
    _same(pac.Result(*[np.concatenate(c) for c in cat], None), one.edges, one.tris, one.tets)
