#!/usr/bin/env python
"""Throughput of the weighted alpha complex engine on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (per rank): a 100,000-ball synthetic globule (self-avoiding walk,
0.05 balls/A^3, C/N/O/S radii), solvent radius 1.4, alpha 1.0, upstream
formulas, the empty-orthosphere test applied (as the reference source is
written), strict single-precision arithmetic.  A step is one full pass: balls
in, the sorted edge/triangle/tetrahedron lists out.  Every rank builds its
own molecule (seeded by rank): the work partitions with no collective, so
scaling is weak.

Prints one JSON line (rank 0).  `value` is device-resident throughput
(inputs already in HBM, lists left in HBM); `e2e` goes through the host C ABI
(pac_alpha_complex: host balls in, pinned host lists out, copies inside the
timed region).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

N_BALLS = 100_000
SOL, ALPHA = 1.4, 1.0
METRIC = "balls/s to bit-exact alpha complex at 100k balls"
CPU_SAMPLE = 10_000


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of the tetrahedron kernel from the committed ncu
    summary (profiles/k_tets_*.md, line 'traffic_bytes_per_launch_full: X')."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if f.startswith("k_tets") and f.endswith(".md"):
            for line in open(os.path.join(d, f)):
                if line.strip().startswith("traffic_bytes_per_launch_full:"):
                    try:
                        return float(line.split(":", 1)[1].strip().split()[0])
                    except ValueError:
                        return None
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.f.close()
        except Exception:
            pass

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines()]
            os.unlink(self.path)
        except Exception:
            return None
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_baseline(threads):
    """The CPU restatement (OpenMP, all host threads) on a bounded sample of
    the same workload: a 10,000-ball globule, same sol-rad/alpha/formulas."""
    pac = ge.load_package()
    orc = ge.load_oracle()
    balls = pac.globule(CPU_SAMPLE, seed=pac.SEED_BASE + 4)
    t0 = time.perf_counter()
    orc.alpha_complex(balls, SOL, ALPHA, orc.UPSTREAM, tet_ortho=True, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": CPU_SAMPLE / dt, "unit": "balls/s", "cores": threads, "kind": "port",
            "sample": "%d-ball globule, sol 1.4, alpha 1.0, as-written, %.2f s" % (CPU_SAMPLE, dt)}


GOLDEN = os.path.join(ROOT, "tests", "golden")


def config_of(n):
    size = "100k" if n - 8 == N_BALLS else "%d" % (n - 8)
    return {"workload": size + "-ball globule (0.05/A^3) + 8 isolated corner balls, sol 1.4, "
                        "alpha 1.0, upstream formulas, orthosphere test applied, strict f32",
            "n_balls": n, "sol_rad": SOL, "alpha": ALPHA, "parallelism": "dp1",
            "l2": "flushed between steps (256 MB write)"}


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def _golden(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def reference_binary_record():
    """The reference binary's own run on the full headline workload (one run,
    tests/golden/refrun/refrun_manifest.json, case glob100k_s14_a1, recorded
    by tests/golden/make_refrun_golden.py on a B200)."""
    man = _golden(os.path.join("refrun", "refrun_manifest.json")) or {}
    rec = man.get("glob100k_s14_a1", {}).get("builds", {}).get("rr128-nofma")
    if not rec or rec.get("rc") != 0:
        return None
    head = _golden("headline_100k.json") or {}
    return {"binary": "parallelac-largeData built with -maxrregcount=128 -fmad=false",
            "n_balls": man["glob100k_s14_a1"]["n"], "total_ms": rec.get("total_ms"),
            "wall_s": rec.get("wall_s"),
            "balls_per_s": man["glob100k_s14_a1"]["n"] / (rec["total_ms"] / 1e3)
            if rec.get("total_ms") else None,
            "lists_equal_headline_digest": rec.get("sha256") == head.get("sha256"),
            "on": "one B200, recorded once (tests/golden/refrun/refrun_manifest.json)"}


def run_reference(args):
    """The reference arm.  The reference (AlphaComplexLargeData.cu) is a CUDA
    program with no CPU implementation of the path; its arithmetic and
    decision procedure are restated on the CPU by the oracle
    (oracle/pac_oracle.c, pinned to the reference binary's own outputs), and
    that port is what this arm times: the whole 100,008-ball workload per
    step, all host threads, the same config, metric and unit as the GPU arm.
    The input comes from the oracle library's copy of the workload generator
    (no library of the product is loaded).  The reference binary itself,
    run once on the same workload on a B200 (a few minutes per run), is
    reported beside it as `reference_binary`."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    orc = ge.load_oracle()
    balls = orc.pad_corners(orc.globule(N_BALLS, seed=orc.SEED_BASE + 4))
    n = len(balls)
    head = _golden("headline_100k.json")
    # the restatement has no warm-up effects beyond page faults: one untimed
    # run whatever W is, so that the arm ends within minutes
    for _ in range(min(args.warmup, 1)):
        e, t, q, _ = orc.alpha_complex(balls, SOL, ALPHA, orc.UPSTREAM, tet_ortho=True,
                                       threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e, t, q, _ = orc.alpha_complex(balls, SOL, ALPHA, orc.UPSTREAM, tet_ortho=True,
                                       threads=threads)
        times.append(time.perf_counter() - t0)
    per = sum(times) / len(times)
    v = n / per
    parity = bool(head) and [_sha(e), _sha(t), _sha(q)] == head["sha256"]
    sample = ("the full %d-ball workload per step (CPU restatement of the reference, "
              "%d host threads)" % (n, threads))
    line = {"impl": "reference", "metric": METRIC, "unit": "balls/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": min(args.warmup, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(n), "value": v, "ms_per_step": per * 1e3,
            "cpu_baseline": {"value": v, "unit": "balls/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "balls/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "parity": {"headline_100k": parity},
            "reference_binary": reference_binary_record()}
    print(json.dumps(line), flush=True)
    return 0


def _device_lists(cx):
    """Host copies of a device complex's three lists (through torch)."""
    import ctypes
    import torch

    class _View:
        def __init__(self, ptr, count):
            self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4",
                                             "data": (ptr, False), "version": 2}

    out = []
    for ptr, rows, k in ((cx.edges, cx.n_edges, 2), (cx.tris, cx.n_tris, 3),
                         (cx.tets, cx.n_tets, 4)):
        if rows == 0:
            out.append(np.zeros((0, k), np.uint32))
            continue
        addr = ctypes.cast(ptr, ctypes.c_void_p).value
        t = torch.as_tensor(_View(addr, rows * k), device="cuda")
        out.append(t.cpu().numpy().view(np.uint32).reshape(rows, k))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_BALLS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-molecules", type=int, default=4096)
    ap.add_argument("--queue-entries", type=int, default=0,
                    help="cap the alpha-tetrahedron queue (32 B entries; default: a quarter "
                         "of free device memory, at most 12 GiB), e.g. to keep a profiled "
                         "run's device memory small")
    ap.add_argument("--no-exact", action="store_true",
                    help="skip the decision-exact (precision cascade) measurements")
    ap.add_argument("--no-assembly", action="store_true",
                    help="skip the 2.5M-ball assembly pass reported beside the headline")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    pac = ge.load_package()
    n = args.n
    # the globule plus 8 isolated corner balls (see pad_corners): every window
    # centre then lies inside the grid, so the reference can run this input
    balls = pac.pad_corners(pac.globule(n, seed=pac.SEED_BASE + 4 + 1000 * rank))
    n = len(balls)
    eng = pac.Engine(device=local, formula="upstream", tet_mode="as-written", predicates="strict",
                     queue_entries=args.queue_entries or None)
    d_balls = torch.from_numpy(balls).cuda()
    torch.cuda.synchronize()  # the engine's stream does not wait on torch's
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        cx, st = eng.alpha_complex_device(d_balls.data_ptr(), n, SOL, ALPHA)

    # ---- device-resident timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    stats = []
    sampler = ClockSampler(local)
    barrier()
    with sampler:
        t0 = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev[k][0].record(stream)
            cx, st = eng.alpha_complex_device(d_balls.data_ptr(), n, SOL, ALPHA)
            ev[k][1].record(stream)
            stats.append(st)
        barrier()
        wall = time.perf_counter() - t0
    step_ms = [a.elapsed_time(b) for a, b in ev]

    # ---- parity of the last timed pass: its lists and stage counters
    # against the restatement's digests (tests/golden/headline_100k.json),
    # outside the timed region
    parity = {}
    head = _golden("headline_100k.json")
    if head and rank == 0 and n == head["balls"]:
        E, T, Q = _device_lists(cx)
        s_last = stats[-1]
        parity["headline_100k"] = ([_sha(E), _sha(T), _sha(Q)] == head["sha256"] and
                                   all(s_last[k] == v for k, v in head["stats"].items()))
        del E, T, Q
    dev_ms = sum(step_ms)

    # ---- union volume/area and their gradients on the final complex
    xyzr = torch.from_numpy(pac.grown_radii(balls, SOL, ALPHA)).cuda()
    dvol = torch.empty((n, 4), dtype=torch.float64, device="cuda")
    darea = torch.empty((n, 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    cx, _ = eng.alpha_complex_device(d_balls.data_ptr(), n, SOL, ALPHA)
    for _ in range(2):
        eng.union_measure_device(xyzr.data_ptr(), n, cx, dvol.data_ptr(), darea.data_ptr())
    gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for k in range(args.steps):
        gev[k][0].record(stream)
        uvol, uarea = eng.union_measure_device(xyzr.data_ptr(), n, cx, dvol.data_ptr(),
                                               darea.data_ptr())
        gev[k][1].record(stream)
    torch.cuda.synchronize()
    grad_ms = sum(a.elapsed_time(b) for a, b in gev) / args.steps
    t_max = dev_ms
    if dist:
        t = torch.tensor([dev_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    ms_per_step = t_max / args.steps
    value = world * n / (ms_per_step / 1e3)

    # ---- end-to-end through the host C ABI
    # ms_total: CUDA events on the engine's stream from before the input copy
    # to after the lists have landed in pinned host memory; the host wall time
    # of the Python call (which also copies the lists into numpy) is reported
    # beside it
    e2e_ms, e2e_wall = [], []
    h2d = d2h = 0
    eng.alpha_complex(balls, SOL, ALPHA)
    barrier()
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        r = eng.alpha_complex(balls, SOL, ALPHA)
        e2e_wall.append(time.perf_counter() - t1)
        e2e_ms.append(max(r.stats["ms_total"], 0.0))
        h2d = balls.nbytes
        d2h = r.edges.nbytes + r.tris.nbytes + r.tets.nbytes
    e2e_step = sum(e2e_ms) / len(e2e_ms)
    if dist:
        t = torch.tensor([e2e_step], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_step = float(t.item())
    e2e_value = world * n / (e2e_step / 1e3)

    # ---- the 2.5M-ball assembly (400 globules of 6,250 balls, sol 1.4,
    # alpha 1) in one call, inputs resident in HBM; reported beside the
    # headline, not part of it
    assembly = None
    if not args.no_assembly:
        ab = pac.assembly()
        d_ab = torch.from_numpy(ab).cuda()
        torch.cuda.synchronize()
        for _ in range(2):  # the first sizes the pool, the second settles it
            eng.alpha_complex_device(d_ab.data_ptr(), len(ab), SOL, ALPHA)
        flush.zero_()
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        _, ast = eng.alpha_complex_device(d_ab.data_ptr(), len(ab), SOL, ALPHA)
        a1.record(stream)
        torch.cuda.synchronize()
        ams = a0.elapsed_time(a1)
        apeak = measured_peaks()[0]
        assembly = {
            "balls": int(len(ab)), "ms": ams, "balls_per_s": len(ab) / (ams / 1e3),
            "complex": [ast["final_edges"], ast["final_tris"], ast["final_tets"]],
            "cand_tets": ast["cand_tets"], "alpha_tets": ast["alpha_tets"],
            "stage_ms": {k: round(ast[k], 3) for k in ("ms_grid", "ms_edges", "ms_tris", "ms_tets",
                                                       "ms_tri_attach", "ms_edge_attach", "ms_emit")},
            "tet_stage_roofline_frac": 64.0 * ast["cand_tets"] / (ast["ms_tets"] / 1e3) / 1e9 / apeak,
            "pass_roofline_frac": ast["bytes_model"] / (ams / 1e3) / 1e9 / apeak,
            "what": "one alpha_complex_device call, CUDA events; as written, strict"}
        del d_ab

    # ---- roofline of the dominant stage (enumeration + orthosphere scan)
    s0 = stats[-1]
    tet_ms = sum(s["ms_tets"] for s in stats) / len(stats)
    # reference byte model: every candidate tetrahedron (16 B) and its
    # orthosphere (16 B) written once and read once
    alg_bytes = 64.0 * s0["cand_tets"]
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (tet_ms / 1e3) / 1e9
    traffic = profiled_traffic()

    # ---- batched vs plain per-molecule launches: the 4,096-molecule batch
    # (sizes log-uniform in [200, 20000], 17.5 M balls), sol 1.4, alpha 0.5;
    # --batch-molecules takes a prefix of it
    batched = None
    if args.batch_molecules > 0:
        sizes = pac.batch_sizes(4096)[:args.batch_molecules]
        bballs, boff = pac.batch(sizes)
        eng.alpha_complex_batch(bballs, boff, SOL, 0.5)
        torch.cuda.synchronize()
        # both arms through the Python binding (which copies the lists out of
        # the context's pinned buffer), and beside them the C calls alone;
        # each arm timed twice (host wall clock on a shared host), the faster
        # run of each reported
        rep = {"batched_s": [], "batched_c_s": [], "plain_s": [], "plain_c_s": []}
        bres = plain = None
        for _ in range(2):
            tb = {}
            bres = None
            t1 = time.perf_counter()
            bres, bst = eng.alpha_complex_batch(bballs, boff, SOL, 0.5, timing=tb)
            rep["batched_s"].append(time.perf_counter() - t1)
            rep["batched_c_s"].append(tb["c_call_s"])
            tp, t_plain_c = {}, 0.0
            plain = None
            plain = []
            t1 = time.perf_counter()
            for m in range(len(sizes)):
                plain.append(eng.alpha_complex(bballs[boff[m]:boff[m + 1]], SOL, 0.5, timing=tp))
                t_plain_c += tp["c_call_s"]
            rep["plain_s"].append(time.perf_counter() - t1)
            rep["plain_c_s"].append(t_plain_c)
        t_batch, t_batch_c = min(rep["batched_s"]), min(rep["batched_c_s"])
        t_plain, t_plain_c = min(rep["plain_s"]), min(rep["plain_c_s"])
        same = all(r.counts() == b.counts() and np.array_equal(r.tets, b.tets) and
                   np.array_equal(r.tris, b.tris) and np.array_equal(r.edges, b.edges)
                   for r, b in zip(plain, bres))
        del plain
        bman = _golden("batch_4096.json")
        if bman and len(sizes) == bman["molecules"]:
            import hashlib
            h = [hashlib.sha256() for _ in range(3)]
            for r in bres:
                for k, a in enumerate((r.edges, r.tris, r.tets)):
                    h[k].update(np.ascontiguousarray(a, dtype=np.uint32).tobytes())
            parity["batch_4096"] = [x.hexdigest() for x in h] == bman["sha256_concat"]
        batched = {"molecules": int(len(sizes)), "balls": int(boff[-1]), "sol_rad": SOL,
                   "alpha": 0.5, "batched_ms": t_batch * 1e3, "plain_ms": t_plain * 1e3,
                   "speedup": t_plain / t_batch, "identical_output": bool(same),
                   "c_calls": {"batched_ms": t_batch_c * 1e3, "plain_ms": t_plain_c * 1e3,
                               "speedup": t_plain_c / t_batch_c,
                               "what": "the C calls alone, lists in the context's pinned "
                                       "buffer on return (no copy, no per-call Python)"},
                   "runs_s": {k: [round(x, 4) for x in v] for k, v in rep.items()},
                   "balls_per_s_batched": float(boff[-1]) / t_batch,
                   "batched_engine_ms": bst["ms_total"],
                   "batched_stage_ms": {k: round(bst[k], 3) for k in
                                        ("ms_h2d", "ms_grid", "ms_edges", "ms_tris", "ms_tets",
                                         "ms_tri_attach", "ms_edge_attach", "ms_emit", "ms_d2h")},
                   "what": "host C ABI both ways through the Python binding (wall clock, "
                           "lists copied to numpy): one pac_alpha_complex_batch call vs one "
                           "pac_alpha_complex call per molecule; each arm run twice, the "
                           "faster run of each (runs_s)"}

    # ---- the precision cascade (PAC_PRED_EXACT): every decision exact, an
    # FP64 filter with a running error bound and 640-bit integers where it
    # cannot tell; throughput on the headline workload and on the 25,000-ball
    # lattice-snapped degeneracy case, with the fallback rates
    exact = None
    if not args.no_exact:
        def timed(engine, dptr, count, sol, alpha, reps=3):
            engine.alpha_complex_device(dptr, count, sol, alpha)  # sizes the pool
            ms, st_ = [], None
            for _ in range(reps):
                flush.zero_()
                torch.cuda.synchronize()
                st_ = engine.alpha_complex_device(dptr, count, sol, alpha)[1]
                ms.append(st_["ms_total"])
            return min(ms), st_

        exact = {"what": "PAC_PRED_EXACT: FP64 filter with a running error bound, 640-bit "
                         "integer fallback; fallback_rate = exact_fallbacks / filter_evals"}
        with pac.Engine(device=local, tet_mode="as-written", predicates="exact") as ex:
            ms, st_ = timed(ex, d_balls.data_ptr(), n, SOL, ALPHA)
            exact["headline_100k"] = {
                "ms": ms, "balls_per_s": n / (ms / 1e3), "filter_evals": st_["filter_evals"],
                "exact_fallbacks": st_["exact_fallbacks"],
                "fallback_rate": st_["exact_fallbacks"] / max(1, st_["filter_evals"]),
                "complex": [st_["final_edges"], st_["final_tris"], st_["final_tets"]]}
        snap = pac.snapped_globule(25_000, seed=pac.SEED_BASE + 1)
        d_snap = torch.from_numpy(snap).cuda()
        torch.cuda.synchronize()
        rec = {"balls": len(snap), "sol_rad": SOL, "alpha": ALPHA,
               "workload": "25,000-ball globule, centres snapped to 0.25 A, radii to 0.05 A"}
        for mode in ("strict", "exact"):
            with pac.Engine(device=local, tet_mode="as-written", predicates=mode) as ex:
                ms, st_ = timed(ex, d_snap.data_ptr(), len(snap), SOL, ALPHA)
            rec[mode] = {"ms": ms, "balls_per_s": len(snap) / (ms / 1e3),
                         "sos_calls": st_["sos_calls"],
                         "complex": [st_["final_edges"], st_["final_tris"], st_["final_tets"]]}
            if mode == "exact":
                rec[mode].update(filter_evals=st_["filter_evals"],
                                 exact_fallbacks=st_["exact_fallbacks"],
                                 fallback_rate=st_["exact_fallbacks"] / max(1, st_["filter_evals"]))
        exact["snapped_25k"] = rec
        del d_snap

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(os.cpu_count() or 1)

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    clocks = sampler.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "balls/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": dict(config_of(n), parallelism="dp%d" % world),
        "simplices_per_s": world * (s0["final_edges"] + s0["final_tris"] + s0["final_tets"] + n)
        / (ms_per_step / 1e3),
        "complex": {"edges": s0["final_edges"], "tris": s0["final_tris"], "tets": s0["final_tets"],
                    "cand_tets": s0["cand_tets"], "alpha_tets": s0["alpha_tets"],
                    "insphere_evals": s0["insphere_evals"], "sos_calls": s0["sos_calls"],
                    "early_refuted": s0["early_refuted"], "cert_decisions": s0["cert_decisions"]},
        "stage_ms": {k: s0[k] for k in ("ms_grid", "ms_edges", "ms_tris", "ms_tets",
                                        "ms_tri_attach", "ms_edge_attach", "ms_emit")},
        "union": {"grad_ms": grad_ms, "volume": uvol, "area": uarea,
                  "what": "volume + area + d/d(centre, radius) of both, FP64, over the final complex"},
        "batched": batched,
        "assembly_2p5m": assembly,
        "e2e": {"value": e2e_value, "unit": "balls/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_step,
                "host_wall_ms_per_step": 1e3 * sum(e2e_wall) / len(e2e_wall)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "tetrahedron stage (k_tets_enum light + heavy, k_tets_scan, k_sos_resolve)",
                     "bytes_model": "64 B x candidate tetrahedra (the reference's tetrahedron "
                                    "and orthosphere lists written and read once)",
                     "kernel_ms": tet_ms},
        # the same model over the whole pass (balls in, lists out, every
        # candidate list and orthosphere of the reference written and read once)
        "pass_roofline": {"achieved": s0["bytes_model"] / (ms_per_step / 1e3) / 1e9,
                          "peak": peak, "unit": "GB/s",
                          "frac": s0["bytes_model"] / (ms_per_step / 1e3) / 1e9 / peak,
                          "bytes": s0["bytes_model"]},
        "cpu_baseline": cpu,
        "parity": parity,
        "exact": exact,
        "gpu_launches": int(sum(s["kernels_launched"] for s in stats)),
        "clocks": clocks,
        "wall_s": wall,
        # per timed step: CUDA events around the call, and the engine's own
        # events from its first to its last operation on the stream
        "step_ms": [round(x, 3) for x in step_ms],
        "engine_ms": [round(s_["ms_total"], 3) for s_ in stats],
    }
    print(json.dumps(line), flush=True)
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
