"""The certified insphere filter (parallelac-xmp_b200/csrc/certify.cuh) on
the CPU: built for the host with the oracle's restatement of the reference's
binary32 orient3d/insphere_w (oracle/pac_oracle.c, compiled without FMA
contraction), it must never claim a decision the replay does not make --
on generic tetrahedra, on balls within 1e-3 of the orthosphere, on nearly
flat tetrahedra, on a 0.25 A lattice with equal radii (exact zeros) and
with a centre 0.05 A off the orthocentre -- while still deciding more than
75 % of the random generic cases (skinny random tetrahedra; on molecules the
scan certifies more than 99 % of its decisions)."""
import os
import subprocess

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def harness(tmp_path_factory, orc):
    out = tmp_path_factory.mktemp("cert") / "cert_harness"
    lib = os.path.join(ROOT, "oracle", "_build")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", str(out),
                    os.path.join(ROOT, "tests", "native", "cert_harness.cpp"),
                    "-L", lib, "-loracle", "-Wl,-rpath," + lib], check=True)
    return str(out)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_certified_filter_never_disagrees_with_replay(harness, seed):
    r = subprocess.run([harness, str(seed), "300000"], capture_output=True, text=True, check=True)
    f = r.stdout.split()
    cases, cert, bad, zeros = int(f[1]), int(f[3]), int(f[5]), int(f[7])
    generic, generic_cert = int(f[9]), int(f[11])
    print(r.stdout.strip())
    assert bad == 0
    assert zeros > 0          # the lattice cases reach exact zeros, never certified
    assert cert > 0.2 * cases
    assert generic_cert > 0.75 * generic
