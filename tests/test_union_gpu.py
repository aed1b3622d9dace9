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
    """The north star's check: 100,000-ball globule, sol 1.4, alpha 1, central
    differences at h = 1e-6 A on 1,000 random (ball, coordinate) pairs, the
    complex held fixed; device entry points, so each evaluation is one pass
    of the measure kernels."""
    import torch
    balls = pac.globule(100_000, seed=pac.SEED_BASE + 4)
    rng = np.random.default_rng(11)
    with pac.Engine(tet_mode="as-written") as eng:
        d = torch.from_numpy(balls).cuda()
        cx, _ = eng.alpha_complex_device(d.data_ptr(), len(balls), SOL, ALPHA)
        x = torch.from_numpy(pac.grown_radii(balls, SOL, ALPHA)).cuda()
        dv = torch.empty_like(x)
        da = torch.empty_like(x)
        torch.cuda.synchronize()
        eng.union_measure_device(x.data_ptr(), len(balls), cx, dv.data_ptr(), da.data_ptr())
        torch.cuda.synchronize()
        gv, ga = dv.cpu().numpy(), da.cpu().numpy()
        h = 1e-6
        err_v, err_a = [], []
        for _ in range(1000):
            i, q = int(rng.integers(len(balls))), int(rng.integers(4))
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
            err_v.append(abs((vp - vm) / (2 * h) - gv[i, q]) / max(1.0, abs(gv[i, q])))
            err_a.append(abs((ap - am) / (2 * h) - ga[i, q]) / max(1.0, abs(ga[i, q])))
    ev, ea = np.array(err_v), np.array(err_a)
    print("FD vs adjoint, 1000 coordinates: volume median %.2e p99 %.2e max %.2e; "
          "area median %.2e p99 %.2e max %.2e; above 1e-6: %d / %d"
          % (np.median(ev), np.quantile(ev, 0.99), ev.max(), np.median(ea), np.quantile(ea, 0.99),
             ea.max(), int((ev > 1e-6).sum()), int((ea > 1e-6).sum())))
    # a perturbation of 1e-6 A can cross a tangency of two circles, where
    # the measure has a kink; the bulk agrees to rounding
    assert np.median(ev) < 1e-9 and np.median(ea) < 1e-9
    assert np.quantile(ev, 0.99) < 1e-6 and np.quantile(ea, 0.99) < 1e-6
    assert ev.max() < 1e-3 and ea.max() < 1e-3
