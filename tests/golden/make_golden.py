"""Regenerate the golden fixtures from the reference tree.

Run in a checkout that has the reference mounted (the fixtures are committed,
so the tests never read the reference tree):

    python tests/golden/make_golden.py /path/to/ParallelAC-xmp

For each shipped reference output (output_files/*.txt) this stores the input
balls exactly as the reference parses them (count with %d, balls with %f,
AlphaComplexLargeData.cu:1070-1079) and the edge/triangle/tetrahedron lists
in the file's own order (AlphaComplexLargeData.cu:2028-2050), plus the sha256
of both source files.  The 1grm output file itself is also kept (gzip) for
the byte-for-byte CLI test.
"""
import ctypes
import gzip
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, crd, output file, binary, formula, alpha, sol-rad
    ("1grm_ld_alpha1", "data/1grm.crd", "output_files/1grm_pAC_LD_alpha1.txt",
     "parallelac-largeData", "upstream", 1.0, 0.0),
    ("1grm_plain_alpha1", "data/1grm.crd", "output_files/1grm_pAC_alpha1.txt",
     "parallelac", "plain-xmp", 1.0, 0.0),
    ("1k4c_plain_alpha1", "data/1k4c.crd", "output_files/1k4c_pAC_alpha1.txt",
     "parallelac", "plain-xmp", 1.0, 0.0),
]


def parse_crd(path):
    libc = ctypes.CDLL(None)
    libc.strtof.restype = ctypes.c_float
    libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    toks = open(path, "rb").read().split()
    n = int(toks[0])
    vals = [libc.strtof(t, None) for t in toks[1:1 + 4 * n]]
    return np.array(vals, dtype=np.float32).reshape(n, 4)


def parse_out(path):
    lines = open(path).read().split("\n")
    n, ne, nt, nq = map(int, lines[0].split())
    def block(a, b, k):
        rows = [list(map(int, l.split())) for l in lines[a:b]]
        return np.array(rows, dtype=np.uint32).reshape(-1, k)
    E = block(1 + n, 1 + n + ne, 2)
    T = block(1 + n + ne, 1 + n + ne + nt, 3)
    Q = block(1 + n + ne + nt, 1 + n + ne + nt + nq, 4)
    return n, E, T, Q


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def main(ref):
    manifest = {}
    for name, crd, out, binary, formula, alpha, sol in CASES:
        balls = parse_crd(os.path.join(ref, crd))
        n, E, T, Q = parse_out(os.path.join(ref, out))
        assert n == len(balls)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), balls=balls, edges=E, tris=T, tets=Q)
        manifest[name] = {"crd": crd, "crd_sha256": sha(os.path.join(ref, crd)), "output": out,
                          "output_sha256": sha(os.path.join(ref, out)), "binary": binary,
                          "formula": formula, "alpha": alpha, "sol_rad": sol,
                          "counts": [int(n), len(E), len(T), len(Q)]}
    with open(os.path.join(ref, "output_files/1grm_pAC_LD_alpha1.txt"), "rb") as f:
        with gzip.open(os.path.join(HERE, "1grm_ld_alpha1.txt.gz"), "wb") as g:
            g.write(f.read())
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_TREE")
    main(sys.argv[1])
