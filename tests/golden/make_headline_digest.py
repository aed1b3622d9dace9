"""Digests of the restatement's complexes for the two workloads the bench
reports, so that the GPU tests and the bench can check the engine on them
without running the CPU restatement on the GPU host:

  headline_100k.json  the 100,000-ball globule (seed SEED_BASE + 4) plus 8
                      isolated corner balls, sol 1.4, alpha 1, upstream
                      formulas, orthosphere test applied: the lists in the
                      reference's output order and the six stage counters.
  batch_4096.json     the 4,096 molecules of log-uniform size in
                      [200, 20000] (17.47 M balls), sol 1.4, alpha 0.5, same
                      options: per molecule the three list lengths, and one
                      sha256 per list kind over all molecules' lists
                      concatenated in molecule order (a checksum over the
                      per-molecule lists; a mismatch is located through the
                      lengths).

    python tests/golden/make_headline_digest.py [headline|batch|all] [--procs P]

The batch runs the molecules in a spawn-started process pool, one thread
each (about 40 minutes on 8 cores)."""
import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SOL = 1.4


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


STAGES = ("cand_edges", "alpha_edges", "cand_tris", "alpha_tris", "cand_tets", "alpha_tets")


def headline():
    import __graft_entry__ as ge
    pac, orc = ge.load_package(), ge.load_oracle()
    balls = pac.pad_corners(pac.globule(100_000, seed=pac.SEED_BASE + 4))
    t0 = time.time()
    e, t, q, st = orc.alpha_complex(balls, SOL, 1.0, orc.UPSTREAM, tet_ortho=True)
    out = {"workload": "100,000-ball globule (seed SEED_BASE + 4) + 8 corner balls, sol 1.4, "
                       "alpha 1.0, upstream formulas, orthosphere test applied",
           "balls": int(len(balls)), "sol_rad": SOL, "alpha": 1.0,
           "input_sha256": hashlib.sha256(balls.tobytes()).hexdigest(),
           "counts": [len(e), len(t), len(q)], "sha256": [sha(e), sha(t), sha(q)],
           "stats": {k: st[k] for k in STAGES},
           "cpu_s": round(time.time() - t0, 1)}
    with open(os.path.join(HERE, "headline_100k.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("headline", out["counts"], out["cpu_s"], "s", flush=True)


_BALLS = None
_OFF = None


def _init(balls, off):
    global _BALLS, _OFF
    _BALLS, _OFF = balls, off


def _molecule(m):
    import __graft_entry__ as ge
    orc = ge.load_oracle()
    b = _BALLS[int(_OFF[m]):int(_OFF[m + 1])]
    e, t, q, _ = orc.alpha_complex(b, SOL, 0.5, orc.UPSTREAM, tet_ortho=True, threads=1)
    return m, e, t, q


def batch(procs):
    import __graft_entry__ as ge
    pac = ge.load_package()
    ge.load_oracle().lib()  # built before the workers start
    sizes = pac.batch_sizes(4096)
    balls, off = pac.batch(sizes)
    t0 = time.time()
    h = [hashlib.sha256() for _ in range(3)]
    counts = []
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=_init, initargs=(balls, off)) as pool:
        for m, e, t, q in pool.imap(_molecule, range(len(sizes)), chunksize=4):
            for k, a in enumerate((e, t, q)):
                h[k].update(np.ascontiguousarray(a, dtype=np.uint32).tobytes())
            counts.append([len(e), len(t), len(q)])
            if m % 256 == 0:
                print("molecule", m, round(time.time() - t0), "s", flush=True)
    c = np.array(counts, dtype=np.int64)
    out = {"workload": "4,096 molecules, sizes log-uniform in [200, 20000] (seed SEED_BASE + 3), "
                       "sol 1.4, alpha 0.5, upstream formulas, orthosphere test applied",
           "molecules": int(len(sizes)), "balls": int(off[-1]), "sol_rad": SOL, "alpha": 0.5,
           "input_sha256": hashlib.sha256(balls.tobytes()).hexdigest(),
           "totals": [int(x) for x in c.sum(0)],
           "sha256_concat": [x.hexdigest() for x in h],
           "edges_per_molecule": [int(x) for x in c[:, 0]],
           "tris_per_molecule": [int(x) for x in c[:, 1]],
           "tets_per_molecule": [int(x) for x in c[:, 2]],
           "cpu_s": round(time.time() - t0, 1), "procs": procs}
    with open(os.path.join(HERE, "batch_4096.json"), "w") as f:
        json.dump(out, f)
    print("batch", out["totals"], out["cpu_s"], "s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", nargs="?", default="all", choices=["headline", "batch", "all"])
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    if a.what in ("headline", "all"):
        headline()
    if a.what in ("batch", "all"):
        batch(a.procs)


if __name__ == "__main__":
    main()
