"""Digests of the restatement's complex for the 2.5M-ball assembly (400
globules of 6,250 balls in an 8 x 10 x 5 grid at 60 A pitch, sol 1.4,
alpha 1), in the reference's output order, with the orthosphere test
applied (as run, every alpha tetrahedron is kept: 6.7 G of them, too many
to hold), so that the GPU test can check the engine at full size without
running the CPU restatement on the GPU host (about 7 minutes on 8 cores):

    python tests/golden/make_assembly_digest.py

writes tests/golden/assembly_2p5m.json."""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import __graft_entry__ as ge  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def main():
    pac, orc = ge.load_package(), ge.load_oracle()
    balls = pac.assembly()
    out = {"balls": int(len(balls)), "sol_rad": 1.4, "alpha": 1.0,
           "input_sha256": hashlib.sha256(balls.tobytes()).hexdigest()}
    t0 = time.time()
    e, t, q, st = orc.alpha_complex(balls, 1.4, 1.0, orc.UPSTREAM, tet_ortho=True)
    out["as-written"] = {"counts": [len(e), len(t), len(q)], "sha256": [sha(e), sha(t), sha(q)],
                         "stats": {k: v for k, v in st.items() if isinstance(v, int)},
                         "cpu_s": round(time.time() - t0, 1)}
    print(out["as-written"]["counts"], out["as-written"]["cpu_s"], flush=True)
    with open(os.path.join(HERE, "assembly_2p5m.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
