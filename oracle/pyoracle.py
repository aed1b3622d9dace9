"""ctypes binding of the CPU restatement (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the bench's cpu_baseline leg, as the checker.  The product path never
imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PRED_PATH = os.path.join(HERE, "_ref", "libpredref.so")

UPSTREAM, PLAIN_XMP = 0, 1
TET_ORTHO = 1  # flag: apply the empty-orthosphere test as written
EXACT = 2      # flag: decision-exact predicates (multi-word integers)


class _Res(ctypes.Structure):
    _fields_ = ([("n_edges", ctypes.c_uint64), ("n_tris", ctypes.c_uint64),
                 ("n_tets", ctypes.c_uint64)] +
                [(k, ctypes.POINTER(ctypes.c_uint32)) for k in ("edges", "tris", "tets")] +
                [(k, ctypes.c_uint64) for k in
                 ("cand_edges", "alpha_edges", "cand_tris", "alpha_tris", "cand_tets",
                  "alpha_tets", "tris_in_tets", "edges_in_tris", "insphere_evals", "sos_calls",
                  "sos_exhausted", "ortho_out_of_grid")] +
                [("grid", ctypes.c_int32 * 3), ("step", ctypes.c_float), ("status", ctypes.c_int)])


_LIB = None


def build():
    """Compile the restatement with its Makefile (gcc, -ffp-contract=off)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_alpha_complex.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(_Res)]
        L.orc_free.argtypes = [ctypes.POINTER(_Res)]
        f3 = ctypes.POINTER(ctypes.c_float)
        L.orc_orient3d.restype = ctypes.c_float
        L.orc_orient3d.argtypes = [f3] * 4
        L.orc_insphere_w.restype = ctypes.c_float
        L.orc_insphere_w.argtypes = [f3] * 5 + [ctypes.c_float] * 5
        L.orc_sos4.restype = ctypes.c_int
        L.orc_sos4.argtypes = [f3] * 5 + [ctypes.c_float] * 5 + [ctypes.c_int] * 5 + [
            ctypes.POINTER(ctypes.c_int)]
        L.orc_exact_pred.restype = ctypes.c_int
        L.orc_exact_pred.argtypes = [ctypes.c_int, f3, ctypes.c_float]
        _LIB = L
    return _LIB


def _take(ptr, count, k):
    if count == 0:
        return np.zeros((0, k), np.uint32)
    return np.ctypeslib.as_array(ptr, (count * k,)).reshape(count, k).copy()


def alpha_complex(balls, sol_rad, alpha, variant=UPSTREAM, tet_ortho=True, threads=0,
                  exact=False):
    """Returns (edges, tris, tets, stats) in the reference binary's order.
    exact=True: decision-exact predicates instead of the reference's
    single-precision formulas."""
    b = np.ascontiguousarray(balls, dtype=np.float32)
    r = _Res()
    flags = (TET_ORTHO if tet_ortho else 0) | (EXACT if exact else 0)
    rc = lib().orc_alpha_complex(b.ctypes.data_as(ctypes.c_void_p), len(b), float(sol_rad),
                                 float(alpha), variant, flags, threads, ctypes.byref(r))
    if rc != 0 or r.status != 0:
        lib().orc_free(ctypes.byref(r))
        raise RuntimeError("oracle failed: %d / status %d" % (rc, r.status))
    try:
        E, T, Q = _take(r.edges, r.n_edges, 2), _take(r.tris, r.n_tris, 3), _take(r.tets, r.n_tets, 4)
        st = {k: int(getattr(r, k)) for k in
              ("cand_edges", "alpha_edges", "cand_tris", "alpha_tris", "cand_tets", "alpha_tets",
               "tris_in_tets", "edges_in_tris", "insphere_evals", "sos_calls", "sos_exhausted",
               "ortho_out_of_grid")}
        st["grid"] = list(r.grid)
        st["step"] = float(r.step)
        return E, T, Q, st
    finally:
        lib().orc_free(ctypes.byref(r))


def _fp(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def orient3d(pa, pb, pc, pd):
    keep = [_fp(p) for p in (pa, pb, pc, pd)]
    return lib().orc_orient3d(*[k[1] for k in keep])


def insphere_w(pa, pb, pc, pd, pe, wa, wb, wc, wd, we):
    keep = [_fp(p) for p in (pa, pb, pc, pd, pe)]
    return lib().orc_insphere_w(*[k[1] for k in keep], wa, wb, wc, wd, we)


def sos4(pts, ws, idx):
    keep = [_fp(p) for p in pts]
    d = ctypes.c_int()
    s = lib().orc_sos4(*[k[1] for k in keep], *[float(w) for w in ws], *[int(i) for i in idx],
                       ctypes.byref(d))
    return s, d.value


def exact_pred(kind, balls, alpha=0.0):
    """One decision-exact predicate on up to five balls (x, y, z, r), weights
    r^2: kind 0 edge alpha, 1 triangle alpha, 2 tetrahedron alpha (2 when
    flat), 3 orient3d sign, 4 insphere sign, 5 edge attached by ball 2,
    6 triangle attached by ball 3."""
    b = np.zeros((5, 4), np.float32)
    a = np.asarray(balls, np.float32)
    b[:len(a)] = a
    return lib().orc_exact_pred(int(kind), b.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                float(alpha))


SEED_BASE = 0xA1FA0000


def globule(n, seed=SEED_BASE):
    """The seeded self-avoiding-walk globule (the workload generator,
    compiled into this library too, so that the checker needs nothing of
    the product's)."""
    L = lib()
    L.pac_synth_globule.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p]
    out = np.zeros((n, 4), np.float32)
    if L.pac_synth_globule(seed, n, out.ctypes.data) != 0:
        raise MemoryError("generator allocation failed")
    return out


def pad_corners(balls, margin=12.0, radius=1.7):
    """balls plus 8 isolated balls at the corners of their bounding box grown
    by `margin` A (the bench's padding; see the package's pad_corners)."""
    b = np.asarray(balls, dtype=np.float32)
    lo = b[:, :3].min(0) - margin
    hi = b[:, :3].max(0) + margin
    corners = [[(lo, hi)[i][0], (lo, hi)[j][1], (lo, hi)[k][2], radius]
               for i in (0, 1) for j in (0, 1) for k in (0, 1)]
    return np.concatenate([b, np.array(corners, np.float32)])


def canonical(a):
    """Sort vertices within each simplex, then the rows lexicographically."""
    a = np.sort(np.asarray(a, dtype=np.int64), axis=1)
    if len(a) == 0:
        return a
    return a[np.lexsort(a.T[::-1])]


def union_measure(xyzr, edges, tris, tets, grad=True):
    """FP64 union volume/area over the given complex (inclusion-exclusion),
    gradients by forward-mode AD.  xyzr: (n, 4) float64 with radii already
    grown (sqrt(r^2 + alpha)).  Returns vol, area, dvol (n,4), darea (n,4)."""
    L = lib()
    x = np.ascontiguousarray(xyzr, dtype=np.float64)
    E = np.ascontiguousarray(edges, dtype=np.uint32)
    T = np.ascontiguousarray(tris, dtype=np.uint32)
    Q = np.ascontiguousarray(tets, dtype=np.uint32)
    n = len(x)
    vol, area = ctypes.c_double(), ctypes.c_double()
    dv = np.zeros((n, 4)) if grad else None
    da = np.zeros((n, 4)) if grad else None
    P = ctypes.c_void_p
    L.orc_union_measure.argtypes = [P, ctypes.c_uint32, P, ctypes.c_uint64, P, ctypes.c_uint64, P,
                                    ctypes.c_uint64, P, P, P, P]
    L.orc_union_measure(x.ctypes.data, n, E.ctypes.data, len(E), T.ctypes.data, len(T),
                        Q.ctypes.data, len(Q), ctypes.addressof(vol), ctypes.addressof(area),
                        dv.ctypes.data if grad else None, da.ctypes.data if grad else None)
    return vol.value, area.value, dv, da


def grown_balls(balls, sol_rad, alpha):
    """(n, 4) float64: centres and radii sqrt((r + sol)^2 + alpha), with the
    radius sum in single precision as the complex sees it."""
    b = np.asarray(balls, dtype=np.float32)
    r = (b[:, 3] + np.float32(sol_rad)).astype(np.float64)
    out = np.empty((len(b), 4))
    out[:, :3] = b[:, :3]
    out[:, 3] = np.sqrt(r * r + float(alpha))
    return out
