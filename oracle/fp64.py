"""FP64 dense-sample evaluation of a tape with a running error bound — TEST
INFRASTRUCTURE.

Only tests/ use this module, as the checker of the outward-rounding mode: every
interval the level passes compute for a box must contain the tape's exact
value at every point of the box. The exact value is not computable, so each
sample is evaluated in double precision together with a rigorous bound E on
the distance between the computed double and the exact real value of the
tape's function at that point (the tape's float32 constants taken as exact).
An interval [lo, hi] passes at a sample with double value v when

    lo <= v + E   and   v - E <= hi .

The "FP64 excess" of a sample is max(lo - v, v - hi): positive means v itself
lies outside the interval (allowed only up to E).

Error propagation, per instruction (u = 2^-53, the unit roundoff of double;
a, b are the computed operands, ea, eb their bounds, r the computed result):
  ADD / SUB   ea + eb + u|r|
  MUL         |a| eb + |b| ea + ea eb + u|r|
  DIV         (|a| eb + |b| ea) / (|b| (|b| - eb)) + u|r|   (inf if |b| <= eb)
  MIN / MAX   max(ea, eb)                 (both are 1-Lipschitz)
  NEG / COPY  ea
  SQRT        of max(a, 0), the function the interval SQRT bounds
              (interval.comp:105-107): min(sqrt(ea), ea / sqrt(a)) + u r
  EXP         r * expm1(ea) + 2u r        (libm's exp is within 1 ulp)
  SIN / COS   ea + 2u                     (|sin'| <= 1; libm within 1 ulp)
The sum of the terms is multiplied by (1 + 2^-40) so that the rounding of the
bound's own arithmetic cannot make it too small. Tape semantics follow
vulkan/shaders/tape/point.comp:2-63 (slots 0..3 = x, y, z, t; result in
slot 0); min/max pick glm's way, which does not matter for the real value.
"""
from __future__ import annotations

import numpy as np

U = 2.0 ** -53
SAFETY = 1.0 + 2.0 ** -40

OP_CONST, OP_SIN, OP_COS, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MIN, OP_MAX, OP_EXP, OP_NEG, OP_SQRT, OP_COPY = range(13)


def decode(wide):
    """Wide instruction words -> (op, out, a, b, const) arrays."""
    w = np.ascontiguousarray(wide, np.uint64)
    op = (w & np.uint64(0xFF)).astype(np.int64)
    out = ((w >> np.uint64(16)) & np.uint64(0xFFFF)).astype(np.int64)
    a = ((w >> np.uint64(32)) & np.uint64(0xFFFF)).astype(np.int64)
    b = (w >> np.uint64(48)).astype(np.int64)
    const = (w >> np.uint64(32)).astype(np.uint32).view(np.float32).astype(np.float64)
    return op, out, a, b, const


def eval_f64(wide, n_slots: int, pts) -> tuple[np.ndarray, np.ndarray]:
    """Values and error bounds of the tape at points pts (N, 4) = (x, y, z, t)
    in double precision. Returns (v, E), each of shape (N,)."""
    pts = np.asarray(pts, np.float64).reshape(-1, 4)
    n = len(pts)
    op, out, ia, ib, const = decode(wide)
    n_slots = max(int(n_slots), 4, int(out.max(initial=0)) + 1)
    v = [None] * n_slots
    e = [None] * n_slots
    zero = np.zeros(n)
    for s in range(4):
        v[s] = pts[:, s].copy()
        e[s] = zero
    with np.errstate(all="ignore"):
        for j in range(len(op)):
            o = op[j]
            if o == OP_CONST:
                r = np.full(n, const[j])
                er = zero
            else:
                a, ea = v[ia[j]], e[ia[j]]
                if o in (OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MIN, OP_MAX):
                    b, eb = v[ib[j]], e[ib[j]]
                if o == OP_ADD:
                    r = a + b
                    er = (ea + eb + U * np.abs(r)) * SAFETY
                elif o == OP_SUB:
                    r = a - b
                    er = (ea + eb + U * np.abs(r)) * SAFETY
                elif o == OP_MUL:
                    r = a * b
                    er = (np.abs(a) * eb + np.abs(b) * ea + ea * eb + U * np.abs(r)) * SAFETY
                elif o == OP_DIV:
                    r = a / b
                    ab = np.abs(b)
                    er = np.where(ab > eb, (np.abs(a) * eb + ab * ea) / (ab * (ab - eb)) + U * np.abs(r),
                                  np.inf) * SAFETY
                elif o == OP_MIN:
                    r = np.where(b < a, b, a)
                    er = np.maximum(ea, eb)
                elif o == OP_MAX:
                    r = np.where(a < b, b, a)
                    er = np.maximum(ea, eb)
                elif o == OP_NEG:
                    r = -a
                    er = ea
                elif o == OP_SQRT:
                    ap = np.maximum(a, 0.0)
                    r = np.sqrt(ap)
                    lip = np.where(ap > 0.0, ea / np.sqrt(np.where(ap > 0.0, ap, 1.0)), np.inf)
                    er = (np.minimum(np.sqrt(ea), lip) + U * r) * SAFETY
                elif o == OP_EXP:
                    r = np.exp(a)
                    er = (r * np.expm1(ea) + 2.0 * U * r) * SAFETY
                elif o == OP_SIN:
                    r = np.sin(a)
                    er = (ea + 2.0 * U) * SAFETY
                elif o == OP_COS:
                    r = np.cos(a)
                    er = (ea + 2.0 * U) * SAFETY
                else:  # COPY
                    r = a
                    er = ea
            v[out[j]] = r
            e[out[j]] = er
    return v[0], e[0]


def box_samples(boxes, per_axis: int = 9, t: float = 0.0) -> np.ndarray:
    """Dense samples of boxes (M, 6) = (low xyz, high xyz): a per_axis^3 grid
    including the corners (per_axis >= 2). Returns (M, per_axis^3, 4)."""
    boxes = np.asarray(boxes, np.float64).reshape(-1, 6)
    s = np.linspace(0.0, 1.0, per_axis)
    gx, gy, gz = np.meshgrid(s, s, s, indexing="ij")
    f = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], -1)          # (P, 3)
    lo, hi = boxes[:, None, :3], boxes[:, None, 3:]
    p = lo + f[None] * (hi - lo)
    # the far face exactly at the high bound (no rounding inside the box edge)
    p = np.where(f[None] == 1.0, np.broadcast_to(hi, p.shape), p)
    tt = np.full(p.shape[:-1] + (1,), float(t))
    return np.concatenate([p, tt], -1)


class Containment:
    """Running summary of interval-vs-FP64 checks."""

    def __init__(self):
        self.samples = 0
        self.skipped = 0            # non-finite double values (e.g. 0/0)
        self.max_excess = -np.inf   # max(lo - v, v - hi) over finite samples
        self.max_err = 0.0          # largest FP64 error bound E seen
        self.max_rel_err = 0.0      # E / max(|v|, 1)
        self.violations = 0         # samples with lo > v + E or v - E > hi
        self.example = None

    def add(self, iv, v, E):
        """iv: (M, 2) intervals; v, E: (M, P) double values and bounds."""
        iv = np.asarray(iv, np.float64)
        lo, hi = iv[:, :1], iv[:, 1:2]
        fin = np.isfinite(v) & np.isfinite(E)
        self.samples += int(fin.sum())
        self.skipped += int((~fin).sum())
        if not fin.any():
            return
        exc = np.maximum(lo - v, v - hi)
        self.max_excess = max(self.max_excess, float(np.max(exc[fin])))
        self.max_err = max(self.max_err, float(np.max(E[fin])))
        self.max_rel_err = max(self.max_rel_err, float(np.max((E / np.maximum(np.abs(v), 1.0))[fin])))
        bad = fin & ((lo > v + E) | (v - E > hi))
        nb = int(bad.sum())
        if nb and self.example is None:
            m, p = np.argwhere(bad)[0]
            self.example = (int(m), int(p), float(lo[m, 0]), float(hi[m, 0]), float(v[m, p]), float(E[m, p]))
        self.violations += nb

    def summary(self) -> dict:
        return {"samples": self.samples, "skipped_nonfinite": self.skipped,
                "max_fp64_excess": self.max_excess, "max_fp64_error_bound": self.max_err,
                "max_fp64_rel_error_bound": self.max_rel_err, "violations": self.violations,
                "example": self.example}


def check_boxes(wide, n_slots, boxes, intervals, t=0.0, per_axis=9, chunk=4096, summary=None) -> Containment:
    """Checks intervals (M, 2) of the tape over boxes (M, 6) against FP64
    samples. Accumulates into `summary` (a Containment) and returns it."""
    summary = summary or Containment()
    boxes = np.asarray(boxes).reshape(-1, 6)
    intervals = np.asarray(intervals).reshape(-1, 2)
    step = max(1, chunk // (per_axis ** 3) * 64)
    for i in range(0, len(boxes), step):
        pts = box_samples(boxes[i:i + step], per_axis, t)
        M, P = pts.shape[:2]
        v, E = eval_f64(wide, n_slots, pts.reshape(-1, 4))
        summary.add(intervals[i:i + step], v.reshape(M, P), E.reshape(M, P))
    return summary
