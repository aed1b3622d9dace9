"""Python binding of libpac (the B200 weighted alpha complex engine).

The directory name is not a Python identifier, so load it by path::

    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "parallelac_xmp_b200", "parallelac-xmp_b200/__init__.py")

(``__graft_entry__.load_package()`` does exactly that.)

Everything here is a thin ctypes layer over ``include/pac.h``; the work runs
in ``lib/libpac.so``.  There is no Python or CPU fallback: if the library or a
CUDA device is missing, the calls raise.
"""
import ctypes
import time
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpac.so")
SYNTH_PATH = os.path.join(HERE, "lib", "libpac_synth.so")
BIN_DIR = os.path.join(HERE, "bin")

FORMULA = {"upstream": 0, "plain-xmp": 1}
TET_MODE = {"as-written": 0, "as-run": 1}
PREDICATES = {"strict": 0, "fma": 1, "exact": 2}
ORDER = {"reference": 0, "canonical": 1}


class PacError(RuntimeError):
    def __init__(self, status, detail):
        super().__init__("%s (%d): %s" % (_lib().pac_status_string(status).decode(), status, detail))
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("formula", ctypes.c_int), ("tet_mode", ctypes.c_int),
                ("predicates", ctypes.c_int), ("order", ctypes.c_int), ("autotune", ctypes.c_int),
                ("verbose", ctypes.c_int), ("reserved_i", ctypes.c_int * 9),
                ("reserved_u", ctypes.c_uint64 * 8)]


class Complex(ctypes.Structure):
    _fields_ = [("n_vertices", ctypes.c_uint32), ("on_device", ctypes.c_uint32),
                ("n_edges", ctypes.c_uint64), ("n_tris", ctypes.c_uint64),
                ("n_tets", ctypes.c_uint64),
                ("edges", ctypes.POINTER(ctypes.c_uint32)),
                ("tris", ctypes.POINTER(ctypes.c_uint32)),
                ("tets", ctypes.POINTER(ctypes.c_uint32))]


class BatchComplex(ctypes.Structure):
    _fields_ = [("n_mol", ctypes.c_uint32), ("on_device", ctypes.c_uint32),
                ("edge_off", ctypes.POINTER(ctypes.c_uint64)),
                ("tri_off", ctypes.POINTER(ctypes.c_uint64)),
                ("tet_off", ctypes.POINTER(ctypes.c_uint64)),
                ("edges", ctypes.POINTER(ctypes.c_uint32)),
                ("tris", ctypes.POINTER(ctypes.c_uint32)),
                ("tets", ctypes.POINTER(ctypes.c_uint32))]


_STAT_U64 = ["n_balls", "n_cells", "cand_edges", "alpha_edges", "cand_tris", "alpha_tris",
             "cand_tets", "alpha_tets", "final_edges", "final_tris", "final_tets",
             "insphere_evals", "sos_calls", "exact_fallbacks", "filter_evals",
             "ortho_out_of_grid", "max_degree"]
_STAT_U64B = ["early_refuted", "early_tests", "cert_decisions", "cert_disagreements"]
_STAT_F64 = ["ms_total", "ms_h2d", "ms_grid", "ms_edges", "ms_tris", "ms_tets",
             "ms_tri_attach", "ms_edge_attach", "ms_emit", "ms_d2h"]


class Stats(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_uint64) for k in _STAT_U64] +
                [(k, ctypes.c_double) for k in _STAT_F64] +
                [("bytes_model", ctypes.c_uint64), ("grid", ctypes.c_uint32 * 3),
                 ("step", ctypes.c_float), ("kernels_launched", ctypes.c_uint32)] +
                [(k, ctypes.c_uint64) for k in _STAT_U64B] +
                [("ms_tet_orthosphere", ctypes.c_double)])

    def as_dict(self):
        d = {k: int(getattr(self, k)) for k in _STAT_U64}
        d.update({k: float(getattr(self, k)) for k in _STAT_F64})
        d["bytes_model"] = int(self.bytes_model)
        d["grid"] = list(self.grid)
        d["step"] = float(self.step)
        d["kernels_launched"] = int(self.kernels_launched)
        d.update({k: int(getattr(self, k)) for k in _STAT_U64B})
        d["ms_tet_orthosphere"] = float(self.ms_tet_orthosphere)
        return d


_LIB = None
_SYNTH = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libpac.so is not built (%s); run parallelac-xmp_b200/build.py"
                               % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.pac_status_string.restype = ctypes.c_char_p
        L.pac_status_string.argtypes = [ctypes.c_int]
        L.pac_last_error.restype = ctypes.c_char_p
        L.pac_abi_version.restype = ctypes.c_int
        L.pac_default_options.argtypes = [ctypes.POINTER(Options)]
        L.pac_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(Options)]
        L.pac_destroy.argtypes = [P]
        L.pac_alpha_complex.argtypes = [P, P, ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                        ctypes.POINTER(Complex), ctypes.POINTER(Stats)]
        L.pac_alpha_complex_device.argtypes = L.pac_alpha_complex.argtypes
        L.pac_alpha_complex_batch.argtypes = [P, P, P, ctypes.c_uint32, ctypes.c_float,
                                              ctypes.c_float, ctypes.POINTER(BatchComplex),
                                              ctypes.POINTER(Stats)]
        L.pac_cuda_stream.restype = ctypes.c_void_p
        L.pac_cuda_stream.argtypes = [P]
        L.pac_union_measure.argtypes = [P, P, ctypes.c_uint32, ctypes.POINTER(Complex), P, P, P, P]
        L.pac_union_measure_device.argtypes = L.pac_union_measure.argtypes
        L.pac_union_measure_noalloc.argtypes = L.pac_union_measure.argtypes
        L.pac_free_complex.argtypes = [ctypes.POINTER(Complex)]
        L.pac_free_batch_complex.argtypes = [ctypes.POINTER(BatchComplex)]
        L.pac_read_crd.argtypes = [ctypes.c_char_p, ctypes.POINTER(P),
                                   ctypes.POINTER(ctypes.c_uint32)]
        L.pac_write_complex.argtypes = [ctypes.c_char_p, P, ctypes.c_uint32, ctypes.c_float,
                                        ctypes.POINTER(Complex)]
        _LIB = L
    return _LIB


def lib():
    """The loaded libpac.so (ctypes.CDLL)."""
    return _lib()


def _check(status):
    if status != 0:
        raise PacError(status, _lib().pac_last_error().decode())


_POOL = None
_POOL_PID = None


def _pool():
    """The binding's copy threads, created on first use (and again in a
    forked child, which does not inherit the parent's threads)."""
    global _POOL, _POOL_PID
    if _POOL is None or _POOL_PID != os.getpid():
        _POOL = ThreadPoolExecutor(min(os.cpu_count() or 1, 64))
        _POOL_PID = os.getpid()
    return _POOL


def _copy_many(srcs):
    """Copies of several 1-D arrays.  Results of 4 MB and more are copied in
    slices of 1-32 MB spread over the host's threads (numpy releases the GIL
    while copying; the first touch of the new pages is most of the cost):
    a 100k-ball complex is 27 MB of lists, a batched pass's run to
    gigabytes."""
    threads = min(os.cpu_count() or 1, 64)
    total = sum(a.nbytes for a in srcs)
    if total < (4 << 20) or threads == 1:
        return [a.copy() for a in srcs]
    step_b = min(32 << 20, max(1 << 20, total // (2 * threads)))
    outs, jobs = [], []
    for a in srcs:
        o = np.empty_like(a)
        outs.append(o)
        step = max(1, step_b // max(1, a.itemsize))
        jobs += [(a, o, i, min(len(a), i + step)) for i in range(0, len(a), step)]
    list(_pool().map(lambda j: np.copyto(j[1][j[2]:j[3]], j[0][j[2]:j[3]]), jobs))
    return outs


def _copy(src):
    return _copy_many([src])[0]


def _view(ptr, count, k):
    if count == 0:
        return np.zeros((0,), np.uint32)
    return np.ctypeslib.as_array(ptr, (count * k,))


class Result:
    """One complex: edges (E,2), tris (T,3), tets (Q,4) uint32 arrays of
    0-based input indices, plus the stage counters of the pass."""

    def __init__(self, edges, tris, tets, stats):
        self.edges, self.tris, self.tets, self.stats = edges, tris, tets, stats

    def counts(self):
        return len(self.edges), len(self.tris), len(self.tets)


class Engine:
    """A pac_ctx: one CUDA stream and device memory pool on one device."""

    def __init__(self, device=0, formula="upstream", tet_mode="as-written", predicates="strict",
                 order="reference", verbose=False, queue_entries=None, autotune=False,
                 enum_blocks=None, scan_blocks=None, heavy_blocks=None, unit_rows=None,
                 scan_claim=None, refute=True, verify=False, slab=None):
        L = _lib()
        if L.pac_abi_version() != 2:
            raise RuntimeError("libpac.so ABI %d, this binding expects 2" % L.pac_abi_version())
        o = Options()
        L.pac_default_options(ctypes.byref(o))
        o.device = device
        o.formula = FORMULA[formula]
        o.tet_mode = TET_MODE[tet_mode]
        o.predicates = PREDICATES[predicates]
        o.order = ORDER[order]
        o.verbose = int(verbose)
        if queue_entries:
            o.reserved_u[0] = int(queue_entries)  # alpha-tetrahedron queue size (testing)
        o.autotune = int(bool(autotune))
        # launch-shape overrides (include/pac.h, pac_options.reserved_i)
        for k, v in enumerate((enum_blocks, scan_blocks, heavy_blocks, unit_rows, scan_claim)):
            if v:
                o.reserved_i[k] = int(v)
        o.reserved_i[5] = 0 if refute else 1
        o.reserved_i[6] = 1 if verify else 0
        if slab:  # (rank, world): one slab of a molecule partitioned by cell order
            o.reserved_i[8], o.reserved_i[7] = int(slab[0]), int(slab[1])
        self._ctx = ctypes.c_void_p()
        _check(L.pac_create(ctypes.byref(self._ctx), ctypes.byref(o)))

    def close(self):
        if self._ctx:
            _lib().pac_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self):
        """The engine's cudaStream_t as an int (for torch.cuda.ExternalStream)."""
        return _lib().pac_cuda_stream(self._ctx) or 0

    def alpha_complex(self, balls, sol_rad, alpha, timing=None):
        """balls: (n, 4) float32 (x, y, z, raw radius) on the host.
        timing: optional dict; receives 'c_call_s', the wall time of the C
        call alone (without this wrapper's copy of the lists)."""
        b = np.ascontiguousarray(balls, dtype=np.float32)
        if b.ndim != 2 or b.shape[1] != 4:
            raise ValueError("balls must have shape (n, 4)")
        cx, st = Complex(), Stats()
        t0 = time.perf_counter()
        rc = _lib().pac_alpha_complex(self._ctx, b.ctypes.data_as(ctypes.c_void_p), len(b),
                                      float(sol_rad), float(alpha), ctypes.byref(cx),
                                      ctypes.byref(st))
        if timing is not None:
            timing["c_call_s"] = time.perf_counter() - t0
        _check(rc)
        try:
            E, T, Q = _copy_many([_view(cx.edges, cx.n_edges, 2), _view(cx.tris, cx.n_tris, 3),
                                  _view(cx.tets, cx.n_tets, 4)])
            return Result(E.reshape(-1, 2), T.reshape(-1, 3), Q.reshape(-1, 4), st.as_dict())
        finally:
            _lib().pac_free_complex(ctypes.byref(cx))

    def alpha_complex_device(self, d_balls_ptr, n, sol_rad, alpha):
        """Device-resident input (a device pointer, e.g. a torch tensor's
        data_ptr()); returns (Complex with device pointers, stats).  The
        lists stay valid until the next call on this engine."""
        cx, st = Complex(), Stats()
        _check(_lib().pac_alpha_complex_device(self._ctx, ctypes.c_void_p(d_balls_ptr), n,
                                               float(sol_rad), float(alpha), ctypes.byref(cx),
                                               ctypes.byref(st)))
        return cx, st.as_dict()

    def union_measure(self, xyzr, result, grad=True):
        """Union volume and area of the balls xyzr ((n, 4) float64, grown
        radii) over the complex `result`, and their gradients (n, 4)."""
        return _union(self, xyzr, result, grad)

    def union_measure_device(self, d_xyzr_ptr, n, cx, d_dvol_ptr=0, d_darea_ptr=0):
        """Device variant: d_xyzr_ptr (n x 4 doubles) and the gradient
        buffers are device pointers; cx a Complex with device lists (from
        alpha_complex_device).  Returns (vol, area)."""
        vol, area = ctypes.c_double(), ctypes.c_double()
        _check(_lib().pac_union_measure_device(
            self._ctx, ctypes.c_void_p(d_xyzr_ptr), n, ctypes.byref(cx), ctypes.addressof(vol),
            ctypes.addressof(area), ctypes.c_void_p(d_dvol_ptr or None),
            ctypes.c_void_p(d_darea_ptr or None)))
        return vol.value, area.value

    def union_measure_noalloc(self, d_xyzr_ptr, n, cx, d_dvol_ptr=0, d_darea_ptr=0):
        """As union_measure_device, but nothing is allocated: the library's
        fixed scratch array is used.  Gradient buffers: both or neither."""
        vol, area = ctypes.c_double(), ctypes.c_double()
        _check(_lib().pac_union_measure_noalloc(
            self._ctx, ctypes.c_void_p(d_xyzr_ptr), n, ctypes.byref(cx), ctypes.addressof(vol),
            ctypes.addressof(area), ctypes.c_void_p(d_dvol_ptr or None),
            ctypes.c_void_p(d_darea_ptr or None)))
        return vol.value, area.value

    def alpha_complex_batch(self, balls, offsets, sol_rad, alpha, timing=None):
        """Many molecules back to back; offsets has n_mol + 1 entries.
        Returns a list of Result (molecule-local indices) and the stats.
        timing: optional dict; receives 'c_call_s', the wall time of the C
        call alone (without this wrapper's copy of the lists)."""
        b = np.ascontiguousarray(balls, dtype=np.float32)
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        nm = len(off) - 1
        bc, st = BatchComplex(), Stats()
        t0 = time.perf_counter()
        rc = _lib().pac_alpha_complex_batch(self._ctx, b.ctypes.data_as(ctypes.c_void_p),
                                            off.ctypes.data_as(ctypes.c_void_p), nm,
                                            float(sol_rad), float(alpha), ctypes.byref(bc),
                                            ctypes.byref(st))
        if timing is not None:
            timing["c_call_s"] = time.perf_counter() - t0
        _check(rc)
        try:
            eo = np.ctypeslib.as_array(bc.edge_off, (nm + 1,)).copy()
            to = np.ctypeslib.as_array(bc.tri_off, (nm + 1,)).copy()
            qo = np.ctypeslib.as_array(bc.tet_off, (nm + 1,)).copy()
            E, T, Q = _copy_many([_view(bc.edges, int(eo[-1]), 2), _view(bc.tris, int(to[-1]), 3),
                                  _view(bc.tets, int(qo[-1]), 4)])
            E, T, Q = E.reshape(-1, 2), T.reshape(-1, 3), Q.reshape(-1, 4)
            res = [Result(E[eo[m]:eo[m + 1]], T[to[m]:to[m + 1]], Q[qo[m]:qo[m + 1]], None)
                   for m in range(nm)]
            return res, st.as_dict()
        finally:
            _lib().pac_free_batch_complex(ctypes.byref(bc))


def grown_radii(balls, sol_rad, alpha):
    """(n, 4) float64 balls for the union measure: centres and radii
    sqrt((r + sol)^2 + alpha), the radius sum taken in single precision as
    the complex sees it."""
    b = np.asarray(balls, dtype=np.float32)
    r = (b[:, 3] + np.float32(sol_rad)).astype(np.float64)
    out = np.empty((len(b), 4))
    out[:, :3] = b[:, :3]
    out[:, 3] = np.sqrt(r * r + float(alpha))
    return out


def _union(eng, xyzr, result, grad):
    x = np.ascontiguousarray(xyzr, dtype=np.float64)
    n = len(x)
    E = np.ascontiguousarray(result.edges, dtype=np.uint32)
    T = np.ascontiguousarray(result.tris, dtype=np.uint32)
    Q = np.ascontiguousarray(result.tets, dtype=np.uint32)
    cx = Complex(n, 0, len(E), len(T), len(Q),
                 E.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                 T.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                 Q.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    vol, area = ctypes.c_double(), ctypes.c_double()
    dv = np.zeros((n, 4)) if grad else None
    da = np.zeros((n, 4)) if grad else None
    _check(_lib().pac_union_measure(eng._ctx, x.ctypes.data, n, ctypes.byref(cx),
                                    ctypes.addressof(vol), ctypes.addressof(area),
                                    dv.ctypes.data if grad else None,
                                    da.ctypes.data if grad else None))
    return vol.value, area.value, dv, da


def read_crd(path):
    """(n, 4) float32 balls of a CRD file, parsed like the reference."""
    L = _lib()
    p = ctypes.c_void_p()
    n = ctypes.c_uint32()
    _check(L.pac_read_crd(os.fsencode(path), ctypes.byref(p), ctypes.byref(n)))
    try:
        if n.value == 0:
            return np.zeros((0, 4), np.float32)
        buf = (ctypes.c_float * (4 * n.value)).from_address(p.value)
        return np.frombuffer(buf, dtype=np.float32).reshape(n.value, 4).copy()
    finally:
        ctypes.CDLL(None).free(p)


def write_complex(path, balls, sol_rad, result):
    """Write `result` in the reference's output file format."""
    b = np.ascontiguousarray(balls, dtype=np.float32)
    E = np.ascontiguousarray(result.edges, dtype=np.uint32)
    T = np.ascontiguousarray(result.tris, dtype=np.uint32)
    Q = np.ascontiguousarray(result.tets, dtype=np.uint32)
    cx = Complex(len(b), 0, len(E), len(T), len(Q),
                 E.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                 T.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                 Q.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    _check(_lib().pac_write_complex(os.fsencode(path), b.ctypes.data_as(ctypes.c_void_p), len(b),
                                    float(sol_rad), ctypes.byref(cx)))


# ----------------------------------------------------------------- workloads
def _synth():
    global _SYNTH
    if _SYNTH is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError("libpac_synth.so is not built; run parallelac-xmp_b200/build.py")
        S = ctypes.CDLL(SYNTH_PATH)
        S.pac_synth_globule.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p]
        S.pac_synth_snapped.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_void_p]
        S.pac_synth_assembly.argtypes = [ctypes.c_uint64] + [ctypes.c_uint32] * 4 + [
            ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
        S.pac_synth_batch_sizes.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_uint32, ctypes.c_void_p]
        S.pac_synth_batch.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                                      ctypes.c_void_p]
        _SYNTH = S
    return _SYNTH


SEED_BASE = 0xA1FA0000


def globule(n, seed=SEED_BASE):
    """Self-avoiding-walk globule of n balls at 0.05 balls/A^3."""
    out = np.zeros((n, 4), np.float32)
    if _synth().pac_synth_globule(seed, n, out.ctypes.data) != 0:
        raise MemoryError("generator allocation failed")
    return out


def snapped_globule(n, seed=SEED_BASE + 1, grid=0.25, rq=0.05):
    """Globule with centres on a `grid` lattice and radii quantised to `rq`."""
    out = np.zeros((n, 4), np.float32)
    if _synth().pac_synth_snapped(seed, n, grid, rq, out.ctypes.data) != 0:
        raise MemoryError("generator allocation failed")
    return out


def assembly(nx=8, ny=10, nz=5, per=6250, pitch=60.0, side=57.0, seed=SEED_BASE + 2):
    """nx*ny*nz cube-confined globules on a lattice (the 2.5M-ball assembly)."""
    out = np.zeros((nx * ny * nz * per, 4), np.float32)
    if _synth().pac_synth_assembly(seed, nx, ny, nz, per, pitch, side, out.ctypes.data) != 0:
        raise MemoryError("generator allocation failed")
    return out


def pad_corners(balls, margin=12.0, radius=1.7):
    """balls plus 8 isolated balls at the corners of their bounding box grown
    by `margin` A.  With margin > 2 grid cells the new balls form no
    simplices, and every window centre of the molecule's simplices falls
    inside the grid (the reference reads the centre cell without a range
    check)."""
    b = np.asarray(balls, dtype=np.float32)
    lo = b[:, :3].min(0) - margin
    hi = b[:, :3].max(0) + margin
    corners = [[(lo, hi)[i][0], (lo, hi)[j][1], (lo, hi)[k][2], radius]
               for i in (0, 1) for j in (0, 1) for k in (0, 1)]
    return np.concatenate([b, np.array(corners, np.float32)])


def batch_sizes(count=4096, lo=200, hi=20000, seed=SEED_BASE + 3):
    s = np.zeros(count, np.uint32)
    _synth().pac_synth_batch_sizes(seed, count, lo, hi, s.ctypes.data)
    return s


def batch(sizes, seed=SEED_BASE + 3):
    """Molecules of the given sizes back to back, and their offsets."""
    sizes = np.ascontiguousarray(sizes, dtype=np.uint32)
    off = np.zeros(len(sizes) + 1, np.uint64)
    off[1:] = np.cumsum(sizes.astype(np.uint64))
    out = np.zeros((int(off[-1]), 4), np.float32)
    if _synth().pac_synth_batch(seed, len(sizes), sizes.ctypes.data, out.ctypes.data) != 0:
        raise MemoryError("generator allocation failed")
    return out, off


# ---------------------------------------------------------------- many GPUs
def shard_molecules(sizes, world):
    """Greedy size balance of independent molecules over `world` ranks:
    largest first, each to the least-loaded rank (ties to the lower rank).
    Returns one ascending index array per rank."""
    sizes = np.asarray(sizes, dtype=np.int64)
    load = [0] * world
    parts = [[] for _ in range(world)]
    for m in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(m)
        load[r] += int(sizes[m])
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def _gather_rows(arrays, rank, world, group=None):
    """Rank 0 receives every rank's 2-D uint32 arrays (one list of them per
    rank, in rank order; None elsewhere): the row counts first (one
    all_gather), then each array padded to the largest count (one gather
    each) -- tensors, so NCCL or gloo moves them without pickling."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    counts = torch.tensor([len(a) for a in arrays], dtype=torch.int64, device=dev)
    allc = [torch.zeros_like(counts) for _ in range(world)]
    dist.all_gather(allc, counts, group=group)
    allc = torch.stack(allc).cpu().numpy()
    out = [[] for _ in range(world)] if rank == 0 else None
    for k, a in enumerate(arrays):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        width = a.shape[1]
        rows = int(allc[:, k].max())
        buf = torch.zeros((max(rows, 1), width), dtype=torch.int32, device=dev)
        if len(a):
            buf[:len(a)] = torch.from_numpy(a.view(np.int32)).to(dev)
        recv = [torch.zeros_like(buf) for _ in range(world)] if rank == 0 else None
        dist.gather(buf, recv, dst=0, group=group)
        if rank == 0:
            for r in range(world):
                out[r].append(recv[r][:int(allc[r, k])].cpu().numpy().view(np.uint32))
    return out


def sharded_batch(balls, offsets, rank, world, run, group=None):
    """Many molecules over the ranks of a torch.distributed group: rank r
    computes the molecules shard_molecules() gives it with
    run(balls, offsets) -> [(edges, tris, tets)] (one rank-local batched
    pass, e.g. an Engine's alpha_complex_batch), and rank 0 receives every
    molecule's lists in the original order (None on the other ranks).  The
    molecules are independent: the only collective is the final gather, of
    tensors (each rank's lists concatenated, and per molecule its id and
    row counts)."""
    off = np.asarray(offsets, dtype=np.uint64)
    sizes = np.diff(off.astype(np.int64))
    mine = shard_molecules(sizes, world)[rank]
    if len(mine):
        parts = [np.asarray(balls[off[m]:off[m + 1]]) for m in mine]
        loff = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.uint64)
        res = run(np.concatenate(parts), loff)
    else:
        res = []
    cat = [np.concatenate([np.asarray(r[k], np.uint32).reshape(-1, w) for r in res])
           if len(res) else np.zeros((0, w), np.uint32) for k, w in enumerate((2, 3, 4))]
    meta = np.array([[m] + [len(r[k]) for k in range(3)] for m, r in zip(mine, res)],
                    np.uint32).reshape(-1, 4)
    got = _gather_rows(cat + [meta], rank, world, group)
    if rank != 0:
        return None
    out = [None] * len(sizes)
    for r in range(world):
        E, T, Q, M = got[r]
        at = [0, 0, 0]
        for m, ne, nt, nq in M:
            cnt = (int(ne), int(nt), int(nq))
            out[int(m)] = tuple(x[at[k]:at[k] + cnt[k]] for k, x in enumerate((E, T, Q)))
            at = [at[k] + cnt[k] for k in range(3)]
    return out


def slab_cuts(balls, sol_rad, alpha, world):
    """The partition of one molecule that Engine(slab=(r, world)) uses, on
    the host: the cell-sorted order of the balls (the reference's stable
    sort by cell key, AlphaComplexLargeData.cu:65-78, 1174-1177; binary32
    arithmetic as there) and the cuts [own_lo, own_hi) of each rank -- ball
    positions n r / world rounded down to the start of their cell.  Returns
    (order, cuts): order[k] is the input index of the k-th ball in cell
    order, cuts has world + 1 entries."""
    b = np.asarray(balls, dtype=np.float32)
    n = len(b)
    with np.errstate(all="ignore"):
        lo = b[:, :3].min(0)
        mr = b[:, 3].max()
        step = np.float32(2.0) * np.sqrt(np.float32(mr * mr + np.float32(alpha)), dtype=np.float32)
        ext = b[:, :3].max(0) - lo
        g = (ext / step).astype(np.int64) + 1
        c = ((b[:, :3] - lo) / step).astype(np.int64)
    key = c[:, 0] + g[0] * c[:, 1] + g[0] * g[1] * c[:, 2]
    order = np.argsort(key, kind="stable")
    skey = key[order]
    cuts = [0]
    for r in range(1, world):
        t = n * r // world
        cuts.append(int(np.searchsorted(skey, skey[t], side="left")) if t < n else n)
    cuts.append(n)
    for r in range(1, world + 1):  # ranges stay ordered when cells are large
        cuts[r] = max(cuts[r], cuts[r - 1])
    return order, np.array(cuts, dtype=np.int64)


def sharded_slab(balls, sol_rad, alpha, rank, world, engine, group=None):
    """One molecule over the ranks of a torch.distributed group: rank r runs
    engine.alpha_complex on its slab (the engine must be made with
    slab=(rank, world)); rank 0 receives the whole complex, the ranks' lists
    concatenated in rank order (None on the other ranks).  Every rank holds
    all the balls; the only collective is the final gather."""
    r = engine.alpha_complex(balls, sol_rad, alpha)
    got = _gather_rows([r.edges, r.tris, r.tets], rank, world, group)
    if rank != 0:
        return None
    return tuple(np.concatenate([got[q][k] for q in range(world)]) for k in range(3))
