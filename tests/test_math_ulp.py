"""Accuracy of the library's transcendentals and of the oracle's directed
rounding, the two facts the outward mode's soundness rests on.

* frep_sinf / frep_cosf / frep_expf (include/frep/frep_math.h) must be within
  one ulp: the outward SIN/COS/EXP intervals widen the function values by one
  float step (frep_next_down / frep_next_up), so the exact value must lie
  strictly between the neighbours of the returned float. Checked against
  x87 long double (64-bit significand: its own error, ~2^-63 relative, is
  ~2^-40 of a float ulp, far inside the margin) on a dense grid and on the
  hard cases: arguments next to multiples of pi/2, the 2^20 reduction limit,
  the exp overflow / underflow / subnormal edges. Host here; the device in
  test_gpu_math_ulp below (same functions, the same bits).
* oracle_directed (the oracle's rounding-mode arithmetic) must give the exact
  result rounded down / up, checked with fractions.Fraction.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np
import pytest

import frep
import oracle
from frep import csg

F32 = np.float32
LD = np.longdouble


def _arguments(kind: str, n_dense: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if kind in ("sin", "cos"):
        dense = rng.uniform(-2.0 ** 20, 2.0 ** 20, n_dense)
        small = rng.uniform(-8.0, 8.0, n_dense // 4)
        tiny = np.exp2(rng.uniform(-140, -1, n_dense // 16)) * rng.choice([-1, 1], n_dense // 16)
        k = np.unique(np.concatenate([np.arange(-64, 65), rng.integers(-667_000, 667_000, 4000)]))
        base = (k.astype(np.float64) * (np.pi / 2)).astype(F32)
        near = [base]
        for s in (1, 2, 3):
            near.append(np.nextafter(near[-1], F32(np.inf)))
        down = [base]
        for s in (1, 2, 3):
            down.append(np.nextafter(down[-1], F32(-np.inf)))
        edge = np.array([2.0 ** 20, -2.0 ** 20, np.nextafter(F32(2.0 ** 20), F32(0)),
                         np.nextafter(F32(-2.0 ** 20), F32(0)), 0.0, -0.0], F32)
        x = np.concatenate([dense.astype(F32), small.astype(F32), tiny.astype(F32), *near, *down, edge])
    else:
        dense = rng.uniform(-104.0, 88.7, n_dense)
        lo_edges = []
        for e in (-87.33654, -103.27893, -103.97208, -149.0, -150.0, 88.72283, 88.0, 0.0):
            c = F32(e)
            lo_edges.append(c)
            u = c
            d = c
            for _ in range(8):
                u = np.nextafter(u, F32(np.inf))
                d = np.nextafter(d, F32(-np.inf))
                lo_edges += [u, d]
        tiny = np.exp2(rng.uniform(-140, -1, n_dense // 16)) * rng.choice([-1, 1], n_dense // 16)
        x = np.concatenate([dense.astype(F32), np.array(lo_edges, F32), tiny.astype(F32)])
    return x.astype(F32)


def _reference(kind: str, x: np.ndarray) -> np.ndarray:
    xl = x.astype(LD)
    return {"sin": np.sin, "cos": np.cos, "exp": np.exp}[kind](xl)


def ulp_check(kind: str, x: np.ndarray, f: np.ndarray) -> dict:
    """Checks that the exact value lies strictly between the neighbours of f
    (with a 2^-40-ulp margin for the long double reference) wherever the
    one-ulp claim applies; returns the worst error in ulps."""
    f = np.asarray(f, F32)
    with np.errstate(all="ignore"):
        ref = _reference(kind, x)
        if kind in ("sin", "cos"):
            claim = np.abs(x.astype(np.float64)) < 2.0 ** 20
            assert np.all(np.abs(f[~claim]) <= 1.0)  # beyond the reduction limit: bounded only
        else:
            # overflow: float infinity stands for values above FLT_MAX
            big = ref > LD(np.finfo(F32).max)
            assert np.all(np.isinf(f[big]))
            claim = ~big
        up = np.nextafter(f, F32(np.inf)).astype(LD)
        dn = np.nextafter(f, F32(-np.inf)).astype(LD)
        fl = f.astype(LD)
        margin = np.abs(ref) * LD(2.0 ** -63) * 4 + LD(2.0 ** -200)
        inside = (ref > dn + margin) & (ref < up - margin)
        step = np.where(ref >= fl, up - fl, fl - dn)
        err = np.abs(ref - fl) / np.where(step > 0, step, LD(1))
    bad = claim & ~inside
    assert not bad.any(), (kind, x[bad][:5], f[bad][:5], ref[bad][:5])
    return {"n": int(claim.sum()), "max_ulp": float(np.max(err[claim]))}


def _tape(kind):
    X = csg.X()
    return frep.Tape({"sin": csg.Sin(X), "cos": csg.Cos(X), "exp": csg.Exp(X)}[kind])


@pytest.mark.parametrize("kind", ["sin", "cos", "exp"])
def test_host_transcendentals_within_one_ulp(kind):
    x = _arguments(kind, 200_000)
    pts = np.zeros((len(x), 4), F32)
    pts[:, 0] = x
    f = _tape(kind).eval_points(pts)
    r = ulp_check(kind, x, f)
    # one rounding of a ~1e-14-accurate double: about half an ulp at worst
    assert r["max_ulp"] < 0.5001, r


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["sin", "cos", "exp"])
def test_gpu_math_ulp(kind):
    """The device's frep_sinf / cosf / expf, through the point interpreter
    (frep_tape_eval_device): within one ulp, and bit-identical to the host."""
    ctx = frep.Context(0, hbm_budget_bytes=2 << 30)
    x = _arguments(kind, 1_000_000, seed=1)
    pts = np.zeros((len(x), 4), F32)
    pts[:, 0] = x
    tape = _tape(kind)
    f = ctx.eval_points(tape, pts)
    r = ulp_check(kind, x, f)
    assert r["max_ulp"] < 0.5001, r
    np.testing.assert_array_equal(f.view(np.uint32), tape.eval_points(pts).view(np.uint32))
    ctx.close()


def _round_dir(q: Fraction, up: bool) -> float:
    fmax = float(np.finfo(F32).max)
    if q > Fraction(fmax):
        return np.inf if up else fmax
    if q < -Fraction(fmax):
        return -fmax if up else -np.inf
    c = F32(float(q))
    while (Fraction(float(c)) < q) if up else (Fraction(float(c)) > q):
        c = np.nextafter(c, F32(np.inf) if up else F32(-np.inf))
    while True:
        n = np.nextafter(c, F32(-np.inf) if up else F32(np.inf))
        if (Fraction(float(n)) >= q) if up else (Fraction(float(n)) <= q):
            c = n
        else:
            return float(c)


def test_oracle_directed_rounding_against_exact_rationals():
    rng = np.random.default_rng(5)
    n = 3000
    mag = np.exp2(rng.uniform(-60, 60, (n, 2))).astype(F32)
    v = (mag * np.where(rng.random((n, 2)) < 0.5, -1, 1)).astype(F32)
    v[:6] = np.array([[1, 3], [0.1, 0.2], [3.4e38, 3.4e38], [-3.4e38, 3.4e38], [1e-40, 3e-41], [7, -0.0]], F32)
    for a, b in v:
        fa, fb = Fraction(float(a)), Fraction(float(b))
        exact = {0: fa + fb, 1: fa - fb, 2: fa * fb}
        if b != 0:
            exact[3] = fa / fb
        for op, q in exact.items():
            assert oracle.directed(op, -1, float(a), float(b)) == _round_dir(q, False), (op, a, b)
            assert oracle.directed(op, +1, float(a), float(b)) == _round_dir(q, True), (op, a, b)
        aa = abs(float(a))
        lo, hi = oracle.directed(4, -1, aa), oracle.directed(4, +1, aa)
        fa = Fraction(aa)
        assert Fraction(lo) ** 2 <= fa < Fraction(float(np.nextafter(F32(lo), F32(np.inf)))) ** 2
        assert fa <= Fraction(hi) ** 2
        assert hi == 0 or Fraction(float(np.nextafter(F32(hi), F32(-np.inf)))) ** 2 < fa
