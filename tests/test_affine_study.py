"""Why the voxelizer has no affine-arithmetic evaluator (the reference's
vulkan/shaders/tape/affine.comp:1-72 is a commented-out sketch): on this
path's scenes a reduced affine form bounds the distance field more loosely
than interval arithmetic, and carrying both gains little.

Both evaluators run here in double precision over the root level's cells
(numpy, one array per slot component), and the test counts the cells each
leaves ambiguous (bounds straddling 0), i.e. the cells that would need
children:
  interval  [lo, hi] per slot, the interval.comp formulas;
  affine    c + ax ex + ay ey + az ez + [-e, e] over the cell's three axes
            (ex, ey, ez in [-1, 1]): linear operations exact, products with
            the quadratic remainder bounded by the product of the radii
            (squares by half of it, centred), decided MIN/MAX passing the
            chosen form through, undecided ones and SQRT falling back to the
            interval hull;
  both      the intersection of the two bounds.
"""
from __future__ import annotations

import numpy as np
import pytest

import frep
from frep import scenes


def _decode(w):
    op, out, a, b = int(w & 0xFF), int((w >> 16) & 0xFFFF), int((w >> 32) & 0xFFFF), int(w >> 48)
    c = float(np.array([int(w >> 32)], np.uint32).view(np.float32)[0])
    return op, out, a, b, c


def _cells(sc, dim):
    cs = sc.world_size / dim
    idx = np.arange(dim ** 3)
    xyz = np.stack([idx // (dim * dim), (idx // dim) % dim, idx % dim], 1).astype(np.float64)
    lo = np.asarray(sc.low_vertex, np.float64) + xyz * cs
    return lo, lo + cs


def _interval(tape, lo, hi, t=0.0):
    n = len(lo)
    S = {0: (lo[:, 0], hi[:, 0]), 1: (lo[:, 1], hi[:, 1]), 2: (lo[:, 2], hi[:, 2]),
         3: (np.full(n, t), np.full(n, t))}
    for w in tape:
        op, o, a, b, c = _decode(w)
        if op == 0:
            S[o] = (np.full(n, c), np.full(n, c))
            continue
        A, B = S[a], S.get(b, S[a])
        if op == 3:
            r = (A[0] + B[0], A[1] + B[1])
        elif op == 4:
            r = (A[0] - B[1], A[1] - B[0])
        elif op == 5:
            p = np.stack([A[0] * B[0], A[0] * B[1], A[1] * B[0], A[1] * B[1]])
            r = (p.min(0), p.max(0))
        elif op == 7:
            r = (np.minimum(A[0], B[0]), np.minimum(A[1], B[1]))
        elif op == 8:
            r = (np.maximum(A[0], B[0]), np.maximum(A[1], B[1]))
        elif op == 10:
            r = (-A[1], -A[0])
        elif op == 11:
            r = (np.sqrt(np.maximum(A[0], 0)), np.sqrt(np.maximum(A[1], 0)))
        elif op == 12:
            r = A
        elif op == 6:  # DIV: A times the reciprocal of B (interval.comp:79-92)
            inv = (1.0 / B[1], 1.0 / B[0])
            p = np.stack([A[0] * inv[0], A[0] * inv[1], A[1] * inv[0], A[1] * inv[1]])
            zero = (B[0] <= 0) & (B[1] >= 0)
            r = (np.where(zero, -np.inf, p.min(0)), np.where(zero, np.inf, p.max(0)))
        elif op == 9:
            r = (np.exp(A[0]), np.exp(A[1]))
        elif op in (1, 2):  # SIN / COS: endpoint values, extrema where a critical point lies inside
            f = np.sin if op == 1 else np.cos
            ph_max, ph_min = (np.pi / 2, -np.pi / 2) if op == 1 else (0.0, np.pi)
            has = lambda ph: np.ceil((A[0] - ph) / (2 * np.pi)) <= np.floor((A[1] - ph) / (2 * np.pi))
            lo_, hi_ = np.minimum(f(A[0]), f(A[1])), np.maximum(f(A[0]), f(A[1]))
            r = (np.where(has(ph_min), -1.0, lo_), np.where(has(ph_max), 1.0, hi_))
        else:
            raise NotImplementedError(op)
        S[o] = r
    return S[0]


def _affine(tape, lo, hi, t=0.0):
    n = len(lo)
    Z = np.zeros(n)
    mid, rad = (lo + hi) / 2, (hi - lo) / 2
    S = {0: (mid[:, 0], rad[:, 0], Z, Z, Z), 1: (mid[:, 1], Z, rad[:, 1], Z, Z),
         2: (mid[:, 2], Z, Z, rad[:, 2], Z), 3: (np.full(n, t), Z, Z, Z, Z)}

    def radius(F):
        return np.abs(F[1]) + np.abs(F[2]) + np.abs(F[3]) + F[4]

    def hull(l, h):
        return ((l + h) / 2, Z, Z, Z, (h - l) / 2)

    for w in tape:
        op, o, a, b, c = _decode(w)
        if op == 0:
            S[o] = (np.full(n, c), Z, Z, Z, Z)
            continue
        A, B = S[a], S.get(b, S[a])
        if op == 3:
            r = tuple(A[i] + B[i] for i in range(4)) + (A[4] + B[4],)
        elif op == 4:
            r = tuple(A[i] - B[i] for i in range(4)) + (A[4] + B[4],)
        elif op == 10:
            r = tuple(-A[i] for i in range(4)) + (A[4],)
        elif op == 12:
            r = A
        elif op == 5:
            ra, rb = radius(A), radius(B)
            if a == b:  # (c + s)^2 = c^2 + 2 c s + s^2, s^2 in [0, ra^2]
                r = (A[0] * A[0] + ra * ra / 2, 2 * A[0] * A[1], 2 * A[0] * A[2], 2 * A[0] * A[3],
                     2 * np.abs(A[0]) * A[4] + ra * ra / 2)
            else:
                r = (A[0] * B[0], A[0] * B[1] + B[0] * A[1], A[0] * B[2] + B[0] * A[2], A[0] * B[3] + B[0] * A[3],
                     np.abs(A[0]) * B[4] + np.abs(B[0]) * A[4] + ra * rb)
        elif op in (7, 8):
            la, ha = A[0] - radius(A), A[0] + radius(A)
            lb, hb = B[0] - radius(B), B[0] + radius(B)
            first, second = (ha < lb, hb < la) if op == 7 else (la > hb, lb > ha)
            fb = hull(np.minimum(la, lb), np.minimum(ha, hb)) if op == 7 else hull(np.maximum(la, lb),
                                                                                    np.maximum(ha, hb))
            r = tuple(np.where(first, A[i], np.where(second, B[i], fb[i])) for i in range(5))
        elif op == 11:
            r = hull(np.sqrt(np.maximum(A[0] - radius(A), 0)), np.sqrt(np.maximum(A[0] + radius(A), 0)))
        elif op in (1, 2, 9):  # linearised at the centre, remainder max|f''| r^2 / 2
            c0, ra = A[0], radius(A)
            if op == 9:
                v, d, m2 = np.exp(c0), np.exp(c0), np.exp(c0 + ra)
            elif op == 1:
                v, d, m2 = np.sin(c0), np.cos(c0), np.ones_like(c0)
            else:
                v, d, m2 = np.cos(c0), -np.sin(c0), np.ones_like(c0)
            r = (v, d * A[1], d * A[2], d * A[3], np.abs(d) * A[4] + m2 * ra * ra / 2)
        elif op == 6:  # A * (1 / B), the reciprocal linearised at B's centre
            cb, rb = B[0], radius(B)
            safe = np.abs(cb) > rb
            m = np.where(safe, np.abs(cb) - rb, 1.0)
            inv = (1.0 / np.where(safe, cb, 1.0), -1.0 / np.where(safe, cb * cb, 1.0))
            Rinv = (inv[0], inv[1] * B[1], inv[1] * B[2], inv[1] * B[3],
                    np.abs(inv[1]) * B[4] + rb * rb / (m ** 3))
            ra, rr = radius(A), radius(Rinv)
            prod = (A[0] * Rinv[0], A[0] * Rinv[1] + Rinv[0] * A[1], A[0] * Rinv[2] + Rinv[0] * A[2],
                    A[0] * Rinv[3] + Rinv[0] * A[3], np.abs(A[0]) * Rinv[4] + np.abs(Rinv[0]) * A[4] + ra * rr)
            inf = np.full_like(cb, np.inf)
            r = tuple(np.where(safe, prod[i], Z if i < 4 else inf) for i in range(5))
        else:
            raise NotImplementedError(op)
        S[o] = r
    F = S[0]
    return F[0] - radius(F), F[0] + radius(F)


@pytest.mark.parametrize("name,make", [("16 spheres", lambda: scenes.spheres_union(16)),
                                       ("64 random primitives", lambda: scenes.random_csg(64, seed=7))])
def test_affine_bounds_are_not_tighter(name, make):
    sc = make()
    tape = frep.Tape(sc.shape).wide()
    lo, hi = _cells(sc, 16)
    il, ih = _interval(tape, lo, hi)
    al, ah = _affine(tape, lo, hi)
    amb_i = int(((il <= 0) & (ih >= 0)).sum())
    amb_a = int(((al <= 0) & (ah >= 0)).sum())
    amb_b = int(((np.maximum(il, al) <= 0) & (np.minimum(ih, ah) >= 0)).sum())
    print(f"{name}: ambiguous root cells of 16^3 -- interval {amb_i}, affine {amb_a}, both {amb_b}")
    assert amb_a >= amb_i            # affine alone is looser
    assert amb_b >= 0.9 * amb_i      # carrying both saves under 10 %
    assert amb_i > 100


def _demo(name, level):
    cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    return scenes.Scene(name, scenes.DEMO_SHAPES[name](level), [16, 4, 4], (-20, -20, -20), 40.0, cam, 64, 48)


def _ambiguous(sc, dim, t):
    tape = frep.Tape(sc.shape).wide()
    lo, hi = _cells(sc, dim)
    with np.errstate(all="ignore"):
        il, ih = _interval(tape, lo, hi, t)
        al, ah = _affine(tape, lo, hi, t)
    return (int(((il <= 0) & (ih >= 0)).sum()), int(((al <= 0) & (ah >= 0)).sum()),
            int(((np.maximum(il, al) <= 0) & (np.minimum(ih, ah) >= 0)).sum()))


# The scenes where affine forms usually pay: transcendentals (the twisted gyroid's
# SIN/COS, the Screw's EXP and rotation by x), rotations that mix axes, and the
# reference's polynomial demo shapes (TangleCube, Morph: x^4 - 8 x^2 terms whose
# interval bounds suffer from the dependency problem). Root cells at 32^3.
WIDER = [("twisted gyroid", lambda: scenes.stress_gyroid(), 0.37, "interval"),
         ("Screw", lambda: _demo("Screw", 0), 2.0, "interval"),
         ("TwistedTower", lambda: _demo("TwistedTower", 4), 0.0, "interval"),
         ("OrganicBalls", lambda: _demo("OrganicBalls", 0), 0.7, "interval"),
         ("TangleCube", lambda: _demo("TangleCube", 0), 0.0, "affine"),
         ("Morph", lambda: _demo("Morph", 0), 0.9, "affine")]


@pytest.mark.parametrize("name,make,t,tighter", WIDER, ids=[w[0] for w in WIDER])
def test_affine_study_wider_scenes(name, make, t, tighter):
    amb_i, amb_a, amb_b = _ambiguous(make(), 32, t)
    print(f"{name}: ambiguous root cells of 32^3 -- interval {amb_i}, affine {amb_a}, both {amb_b}")
    assert amb_b <= min(amb_i, amb_a)
    if tighter == "interval":
        assert amb_i <= amb_a and amb_b >= 0.9 * amb_i
    else:  # the polynomial shapes: affine forms leave under half the ambiguous cells
        assert amb_a < 0.5 * amb_i
