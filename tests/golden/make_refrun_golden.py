"""Run the reference's own binaries (oracle/_ref/, built from the reference
sources by oracle/ref_build.sh) on the parity inputs and record their outputs
as fixtures.  Needs a GPU; run it where the binaries were built or shipped:

    python tests/golden/make_refrun_golden.py OUTDIR [CASE ...]

(no CASE: every case below; OUTDIR/refrun_manifest.json is updated in place,
so cases can be run in separate calls).

Builds used:
    default       AlphaComplexLargeData.cu with nvcc defaults, as the
                  reference's CMakeLists.txt builds it (upstream formulas)
    nofma         ... -fmad=false
    rr128         ... -maxrregcount=128 (checkTetsOrthosphere launches and runs)
    rr128-nofma   both
    plain-rr128, plain-rr128-nofma
                  AlphaComplexParallel.cu (plain-xmp formulas) with the same
                  flags

Safety: the reference reads the window's centre cell without a range check
(AlphaComplexLargeData.cu:625-627, 816-818, 955-957).  Before a binary sees
an input, the CPU restatement evaluates the same windows and the input is
skipped unless no centre index falls outside the grid in either tet mode.

For every (case, build) OUTDIR/refrun_<case>__<build>.npz holds the edge,
triangle and tetrahedron lists in the file's order when they are small, and
OUTDIR/refrun_manifest.json holds counts, sha256 digests of the in-order
lists, and the binary's own "Total time taken (ms)".
"""
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

SMALL_ROWS = 400_000


LD_BUILDS = ["default", "nofma", "rr128", "rr128-nofma"]
PLAIN_BUILDS = ["plain-rr128", "plain-rr128-nofma"]


def cases(pac):
    """(name, balls, sol, alpha, builds, formula of the restatement check)."""
    g = lambda name: np.load(os.path.join(HERE, name + ".npz"))["balls"]
    head = lambda: pac.pad_corners(pac.globule(100_000, seed=pac.SEED_BASE + 4))
    return [
        ("1grm_a1", g("1grm_ld_alpha1"), 0.0, 1.0, LD_BUILDS, 0),
        ("1k4c_a1", g("1k4c_plain_alpha1"), 0.0, 1.0, LD_BUILDS, 0),
        ("glob1300_a0", pac.globule(1300, seed=pac.SEED_BASE), 0.0, 0.0, LD_BUILDS, 0),
        ("snap2000_s14_a1", pac.snapped_globule(2000, seed=pac.SEED_BASE + 1), 1.4, 1.0,
         LD_BUILDS, 0),
        ("glob5000_s14_a1", pac.globule(5000, seed=pac.SEED_BASE + 4), 1.4, 1.0, LD_BUILDS, 0),
        # the plain binary (plain-xmp formulas)
        ("plain_1grm_a1", g("1grm_ld_alpha1"), 0.0, 1.0, PLAIN_BUILDS, 1),
        ("plain_1k4c_a1", g("1k4c_plain_alpha1"), 0.0, 1.0, PLAIN_BUILDS, 1),
        ("plain_glob1300_a0", pac.globule(1300, seed=pac.SEED_BASE), 0.0, 0.0, PLAIN_BUILDS, 1),
        ("plain_glob5000_s14_a1", pac.pad_corners(pac.globule(5000, seed=pac.SEED_BASE + 4)), 1.4,
         1.0, PLAIN_BUILDS, 1),
        ("plain_glob3000_s14_a05", pac.pad_corners(pac.globule(3000, seed=pac.SEED_BASE + 7)),
         1.4, 0.5, PLAIN_BUILDS, 1),
        # the bench's headline workload, one run of the -fmad=false build (a
        # few minutes): its lists pinned, its run time recorded
        ("glob100k_s14_a1", head(), 1.4, 1.0, ["rr128-nofma"], 0),
    ]


def write_crd(path, balls):
    with open(path, "w") as f:
        f.write("%d\n" % len(balls))
        for b in balls:
            f.write("%s %s %s %s\n" % tuple(repr(float(v)) for v in b))


def parse_lists(path):
    with open(path) as f:
        n, ne, nt, nq = map(int, f.readline().split())
        for _ in range(n):
            f.readline()
        E = np.fromstring("".join(f.readline() for _ in range(ne)), dtype=np.int64, sep=" ")
        T = np.fromstring("".join(f.readline() for _ in range(nt)), dtype=np.int64, sep=" ")
        Q = np.fromstring("".join(f.readline() for _ in range(nq)), dtype=np.int64, sep=" ")
    return (E.reshape(-1, 2).astype(np.uint32), T.reshape(-1, 3).astype(np.uint32),
            Q.reshape(-1, 4).astype(np.uint32))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def main(outdir, only=()):
    os.makedirs(outdir, exist_ok=True)
    pac = ge.load_package()
    orc = ge.load_oracle()
    refdir = os.path.join(ROOT, "oracle", "_ref")
    mpath = os.path.join(outdir, "refrun_manifest.json")
    man = json.load(open(mpath)) if os.path.exists(mpath) else {}
    tmp = tempfile.mkdtemp()
    for name, balls, sol, alpha, builds, formula in cases(pac):
        if only and name not in only:
            continue
        oob = 0
        for flag in (False, True):
            if flag is False and len(balls) > 20000:
                continue  # as run, every alpha tetrahedron is kept: too many to hold
            oob += orc.alpha_complex(balls, sol, alpha, formula, tet_ortho=flag)[3][
                "ortho_out_of_grid"]
        entry = {"n": len(balls), "sol_rad": sol, "alpha": alpha, "oob_checked": oob,
                 "formula": "plain-xmp" if formula else "upstream", "builds": {}}
        man[name] = entry
        if oob:
            entry["skipped"] = "window centre outside the grid; the reference would read out of range"
            continue
        crd = os.path.join(tmp, name + ".crd")
        write_crd(crd, balls)
        for b in builds:
            if b.startswith("plain-"):
                exe = os.path.join(refdir, "parallelac-" + b[len("plain-"):])
            else:
                exe = os.path.join(refdir, "parallelac-largeData-" + b if b != "default"
                                   else "parallelac-largeData")
            if not os.path.exists(exe):
                continue
            out = os.path.join(tmp, "%s__%s.txt" % (name, b))
            log = os.path.join(tmp, "%s__%s.log" % (name, b))
            # chunk size >= n: one chunk, no cross-chunk shortcuts (the plain
            # binary takes no chunk size)
            argv = [exe, crd, out, repr(sol), repr(alpha)]
            if not b.startswith("plain-"):
                argv.append(str(len(balls)))
            t0 = time.perf_counter()
            with open(log, "w") as lf:
                r = subprocess.run(argv, stdout=lf, stderr=subprocess.STDOUT, timeout=1200)
            wall = time.perf_counter() - t0
            txt = open(log, errors="replace").read()
            m = re.search(r"Total time taken \(ms\):\s*([0-9.]+)", txt)
            errs = sorted(set(re.findall(r"GPUassert: ([^\n]*)", txt)))
            if r.returncode != 0 or not os.path.exists(out):
                entry["builds"][b] = {"rc": r.returncode, "wall_s": wall, "gpu_errors": errs,
                                      "log_tail": txt[-2000:]}
                continue
            E, T, Q = parse_lists(out)
            rec = {"rc": r.returncode, "wall_s": wall, "total_ms": float(m.group(1)) if m else None,
                   "gpu_errors": errs, "counts": [len(E), len(T), len(Q)],
                   "sha256": [digest(E), digest(T), digest(Q)]}
            if len(E) + len(T) + len(Q) <= SMALL_ROWS:
                np.savez_compressed(os.path.join(outdir, "refrun_%s__%s.npz" % (name, b)),
                                    edges=E, tris=T, tets=Q)
                rec["stored"] = True
            entry["builds"][b] = rec
            os.unlink(out)
        with open(mpath, "w") as f:
            json.dump(man, f, indent=1, sort_keys=True)
    print(json.dumps(man, indent=1, sort_keys=True))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_refrun_golden.py OUTDIR [CASE ...]")
    main(sys.argv[1], tuple(sys.argv[2:]))
