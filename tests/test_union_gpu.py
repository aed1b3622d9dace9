"""Union-of-balls volume and area over the engine's complex, and their
gradients (the hand-written adjoint), against the FP64 CPU oracle (whose
gradients come from forward-mode automatic differentiation) and against
central finite differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOL, ALPHA = 1.4, 1.0


def _setup(pac, n, seed):
    balls = pac.globule(n, seed=seed)
    eng = pac.Engine(tet_mode="as-written")
    r = eng.alpha_complex(balls, SOL, ALPHA)
    return eng, balls, r, pac.grown_radii(balls, SOL, ALPHA)


def test_union_matches_fp64_oracle(pac, orc):
    eng, balls, r, x = _setup(pac, 3000, 31)
    with eng:
        v, a, dv, da = eng.union_measure(x, r)
    ov, oa, odv, oda = orc.union_measure(x, r.edges, r.tris, r.tets)
    assert abs(v - ov) <= 1e-10 * abs(ov)
    assert abs(a - oa) <= 1e-10 * abs(oa)
    # gradients: relative to the largest component of each field
    assert np.abs(dv - odv).max() <= 1e-10 * np.abs(odv).max()
    assert np.abs(da - oda).max() <= 1e-10 * np.abs(oda).max()


def test_union_gradient_central_differences(pac):
    """Central differences at h = 1e-6 A on 40 random coordinates (complex
    held fixed).  Error bound: FD truncation + roundoff ~ 1e-6 relative."""
    eng, balls, r, x = _setup(pac, 1500, 32)
    rng = np.random.default_rng(5)
    h = 1e-6
    with eng:
        v, a, dv, da = eng.union_measure(x, r)
        worst_v = worst_a = 0.0
        for _ in range(40):
            i, q = int(rng.integers(len(x))), int(rng.integers(4))
            xp, xm = x.copy(), x.copy()
            xp[i, q] += h
            xm[i, q] -= h
            vp, ap, _, _ = eng.union_measure(xp, r, grad=False)
            vm, am, _, _ = eng.union_measure(xm, r, grad=False)
            fv, fa = (vp - vm) / (2 * h), (ap - am) / (2 * h)
            worst_v = max(worst_v, abs(fv - dv[i, q]) / max(1.0, abs(dv[i, q])))
            worst_a = max(worst_a, abs(fa - da[i, q]) / max(1.0, abs(da[i, q])))
    print("FD relative error: volume %.2e, area %.2e" % (worst_v, worst_a))
    assert worst_v < 1e-5 and worst_a < 1e-5


def test_union_identity_area_is_volume_radius_derivative(pac):
    eng, balls, r, x = _setup(pac, 800, 33)
    with eng:
        v, a, dv, da = eng.union_measure(x, r)
    assert abs(dv[:, 3].sum() - a) <= 1e-9 * a


@pytest.mark.slow
def test_union_gradient_fd_100k_1000_coordinates(pac):
    """100,000-ball globule, sol 1.4, alpha 1: central differences at
    h = 1e-6 A on 1,000 random (ball, coordinate) pairs, the complex held
    fixed, against the adjoint of one device pass.

    Checked two ways.  (1) On the whole measure through the device entry
    point.  A 1e-6 A step changes the 1.5e6 A^3 total by about 1e-5 A^3,
    while the total itself is a double whose last bit is worth
    ulp(V) = 2.3e-10 A^3; the difference quotient therefore carries up to
    ulp(V) / (2h) = 1.2e-4 of rounding, and the bound is that.  (2) On the
    sub-complex of the simplices that contain the perturbed ball: the
    inclusion-exclusion terms of all other simplices do not depend on the
    ball, so the derivative is the same, and the totals are small enough for
    a tight bound."""
    import torch
    balls = pac.globule(100_000, seed=pac.SEED_BASE + 4)
    rng = np.random.default_rng(11)
    xh = pac.grown_radii(balls, SOL, ALPHA)
    h = 1e-6
    picks = [(int(rng.integers(len(balls))), int(rng.integers(4))) for _ in range(1000)]
    with pac.Engine(tet_mode="as-written") as eng:
        r = eng.alpha_complex(balls, SOL, ALPHA)  # host copy of the lists for (2)
        d = torch.from_numpy(balls).cuda()
        cx, _ = eng.alpha_complex_device(d.data_ptr(), len(balls), SOL, ALPHA)
        assert (cx.n_edges, cx.n_tris, cx.n_tets) == (len(r.edges), len(r.tris), len(r.tets))
        x = torch.from_numpy(xh).cuda()
        dv = torch.empty_like(x)
        da = torch.empty_like(x)
        torch.cuda.synchronize()
        V, A = eng.union_measure_device(x.data_ptr(), len(balls), cx, dv.data_ptr(),
                                        da.data_ptr())
        torch.cuda.synchronize()
        gv, ga = dv.cpu().numpy(), da.cpu().numpy()
        full_v, full_a = [], []
        for i, q in picks:
            # torch writes on its own stream: finish each write before the
            # engine (which launches on another stream) reads the buffer
            x0 = float(x[i, q])
            x[i, q] = x0 + h
            torch.cuda.synchronize()
            vp, ap = eng.union_measure_device(x.data_ptr(), len(balls), cx)
            x[i, q] = x0 - h
            torch.cuda.synchronize()
            vm, am = eng.union_measure_device(x.data_ptr(), len(balls), cx)
            x[i, q] = x0
            torch.cuda.synchronize()
            full_v.append(abs((vp - vm) / (2 * h) - gv[i, q]))
            full_a.append(abs((ap - am) / (2 * h) - ga[i, q]))
        loc_v, loc_a = [], []
        for i, q in picks:
            rows = [L[(L == i).any(axis=1)] for L in (r.edges, r.tris, r.tets)]
            verts = np.unique(np.concatenate([np.array([i], np.uint32)] +
                                             [x_.ravel() for x_ in rows]))
            sub = type("Sub", (), {})()
            sub.edges, sub.tris, sub.tets = (np.searchsorted(verts, L).astype(np.uint32)
                                             for L in rows)
            xl = xh[verts].copy()
            k = int(np.searchsorted(verts, i))
            _, _, lv, la = eng.union_measure(xl, sub)
            xp, xm = xl.copy(), xl.copy()
            xp[k, q] += h
            xm[k, q] -= h
            vp, ap, _, _ = eng.union_measure(xp, sub, grad=False)
            vm, am, _, _ = eng.union_measure(xm, sub, grad=False)
            # the sub-complex adjoint is the full one for this ball
            assert abs(lv[k, q] - gv[i, q]) <= 1e-12 * max(1.0, abs(gv[i, q]))
            assert abs(la[k, q] - ga[i, q]) <= 1e-12 * max(1.0, abs(ga[i, q]))
            loc_v.append(abs((vp - vm) / (2 * h) - gv[i, q]) / max(1.0, abs(gv[i, q])))
            loc_a.append(abs((ap - am) / (2 * h) - ga[i, q]) / max(1.0, abs(ga[i, q])))
    fv, fa, lv_, la_ = map(np.array, (full_v, full_a, loc_v, loc_a))
    ulp_v, ulp_a = np.spacing(V), np.spacing(A)
    print("FD vs adjoint, 1000 coordinates, h = 1e-6 A\n"
          "  whole measure: volume max %.2e (rounding bound %.2e), area max %.2e (bound %.2e)\n"
          "  incident sub-complex, relative: volume median %.2e p99 %.2e max %.2e; "
          "area median %.2e p99 %.2e max %.2e"
          % (fv.max(), ulp_v / h, fa.max(), ulp_a / h, np.median(lv_), np.quantile(lv_, 0.99),
             lv_.max(), np.median(la_), np.quantile(la_, 0.99), la_.max()))
    # (1) two roundings of the total, plus a little for the gradient itself
    assert np.all(fv <= ulp_v / h + 1e-7 * np.maximum(1.0, np.abs(gv[tuple(np.array(picks).T)])))
    assert np.all(fa <= ulp_a / h + 1e-7 * np.maximum(1.0, np.abs(ga[tuple(np.array(picks).T)])))
    # (2) truncation O(h^2) and rounding of totals of a few hundred A^3
    assert np.median(lv_) < 1e-8 and np.median(la_) < 1e-8
    assert np.quantile(lv_, 0.99) < 1e-6 and np.quantile(la_, 0.99) < 1e-6
    assert lv_.max() < 1e-4 and la_.max() < 1e-4


def test_repeated_measure_calls_do_not_grow_device_memory(pac):
    """Each union-measure call copies its inputs and takes its scratch from
    the context's pool and gives them back on return: a loop of a few
    hundred calls (an optimisation or finite-difference loop) leaves the
    device memory in use flat after the first calls."""
    import torch
    balls = pac.globule(1500, seed=34)
    x = pac.grown_radii(balls, SOL, ALPHA)
    with pac.Engine(tet_mode="as-written") as eng:
        r = eng.alpha_complex(balls, SOL, ALPHA)
        d = torch.from_numpy(balls).cuda()
        dx = torch.from_numpy(x).cuda()
        dv = torch.empty_like(dx)
        da = torch.empty_like(dx)
        torch.cuda.synchronize()
        cx, _ = eng.alpha_complex_device(d.data_ptr(), len(balls), SOL, ALPHA)
        for _ in range(3):  # warm: the pool reaches its size for this work
            eng.union_measure(x, r, grad=True)
            eng.union_measure_device(dx.data_ptr(), len(balls), cx, dv.data_ptr(), da.data_ptr())
            eng.union_measure_device(dx.data_ptr(), len(balls), cx)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        first = eng.union_measure_device(dx.data_ptr(), len(balls), cx)
        for _ in range(300):
            eng.union_measure(x, r, grad=True)
            eng.union_measure_device(dx.data_ptr(), len(balls), cx, dv.data_ptr(), da.data_ptr())
            got = eng.union_measure_device(dx.data_ptr(), len(balls), cx)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        # the device complex is still the one computed before the loop
        assert got == first
    assert free0 - free1 < (64 << 20), (free0, free1)
