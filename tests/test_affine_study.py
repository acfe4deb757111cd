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


def _interval(tape, lo, hi):
    n = len(lo)
    S = {0: (lo[:, 0], hi[:, 0]), 1: (lo[:, 1], hi[:, 1]), 2: (lo[:, 2], hi[:, 2]), 3: (np.zeros(n), np.zeros(n))}
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
        else:
            raise NotImplementedError(op)
        S[o] = r
    return S[0]


def _affine(tape, lo, hi):
    n = len(lo)
    Z = np.zeros(n)
    mid, rad = (lo + hi) / 2, (hi - lo) / 2
    S = {0: (mid[:, 0], rad[:, 0], Z, Z, Z), 1: (mid[:, 1], Z, rad[:, 1], Z, Z),
         2: (mid[:, 2], Z, Z, rad[:, 2], Z), 3: (Z, Z, Z, Z, Z)}

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
