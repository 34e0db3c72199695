"""The implicit solver's step-control shortcuts decide exactly what the full computation decides.

The solver kernel (tiger_nga_b200/csrc/bdf_kernel.cuh) skips three computations where cheaper
comparisons already decide their outcome:

* a step-size candidate 1 / (x^(1/e) + 1e-6) is only used when it reaches 1.5, so its power is
  skipped when x > (2/3)^e (1 + 1e-9) (BdfCoef::grow, filled by make_coef in csrc/solver.cu);
* the Newton convergence test x / 0.1 <= 1 (below_tenth) and the Jacobian-refresh test
  |gamma / gamma_lu - 1| > dgmax (gamma_moved) are decided by products with a relative margin
  of 1e-12 and fall back to the division inside that band.

This restates those comparisons in IEEE float64 (numpy) and checks them against the full
computation on values at, just inside and just outside every threshold, plus random values. The
GPU path's own evidence is that the substep's results are bit-identical with and without them.
"""
import numpy as np

KQMAX = 5


def grow(e):
    return (2.0 / 3.0) ** e * (1.0 + 1e-9)


def eta_full(x, e):
    y = 1.0 / e
    return 1.0 / (np.exp(y * np.log(x)) + 1e-6)


def below_tenth(x):
    if x < 0.1 * (1.0 - 1e-12):
        return True
    if x > 0.1 * (1.0 + 1e-12):
        return False
    return x / 0.1 <= 1.0


def gamma_moved(g, glu, dg):
    up, dn = glu * (1.0 + dg), glu * (1.0 - dg)
    if g > up * (1.0 + 1e-12) or g < dn * (1.0 - 1e-12):
        return True
    if g < up * (1.0 - 1e-12) and g > dn * (1.0 + 1e-12):
        return False
    return abs(g / glu - 1.0) > dg


def _around(v, rng, n=2000):
    """Values at and near v: exact neighbours in ulps, relative offsets up to 1e-6, random."""
    out = [v, np.nextafter(v, 0.0), np.nextafter(v, np.inf)]
    k = np.arange(1, 64)
    out += list(v + k * np.spacing(v)) + list(v - k * np.spacing(v))
    rel = np.concatenate([10.0 ** -np.arange(6, 16, 0.25), -(10.0 ** -np.arange(6, 16, 0.25))])
    out += list(v * (1.0 + rel))
    out += list(v * np.exp(rng.uniform(-3, 3, n)))
    return np.array([x for x in out if x > 0.0])


def test_skipped_step_size_candidates_are_below_one_and_a_half():
    rng = np.random.default_rng(20261204)
    for e in range(1, KQMAX + 3):
        thr = grow(e)
        xs = _around(thr, rng)
        skipped = xs[xs > thr]
        assert skipped.size > 0
        eta = eta_full(skipped, e)
        assert np.all(eta < 1.5), (e, skipped[eta >= 1.5][:3])
        # and the threshold is tight: candidates at and above 1.5 exist just below it
        near = xs[(xs <= thr) & (xs > thr * (1 - 1e-3))]
        assert np.any(eta_full(near, e) < 1.5)


def test_convergence_test_matches_the_division():
    rng = np.random.default_rng(7)
    xs = _around(0.1, rng)
    xs = np.concatenate([xs, [0.0, 1e-300, 1e300]])
    for x in xs:
        assert below_tenth(float(x)) == (float(x) / 0.1 <= 1.0), x
    assert below_tenth(float("nan")) is False  # NaN fails the test, as the division does


def test_jacobian_refresh_test_matches_the_division():
    rng = np.random.default_rng(11)
    for dg in (0.3, 0.05, 0.9, 1.5):
        for glu in (1e-12, 3.7e-7, 0.25, 1.0, 123.0):
            for edge in (glu * (1.0 + dg), glu * (1.0 - dg) if dg < 1.0 else glu * 0.5):
                for g in _around(edge, rng, n=500):
                    g = float(g)
                    assert gamma_moved(g, glu, dg) == (abs(g / glu - 1.0) > dg), (g, glu, dg)
    assert gamma_moved(float("nan"), 1.0, 0.3) is False  # NaN compares false either way
