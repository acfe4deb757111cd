"""Tape compiler and host interpreter against the reference (no GPU).

Pins, in order of strength:
* byte-exact equality with the reference's csg::Tape on every golden scene
  (tests/golden/ref_tapes.npz, made by the reference's own compiler) and, when
  the reference tree is present, on freshly generated random scenes;
* bit-exact equality of point evaluation with csg::Tape::Eval on algebraic
  tapes (no SIN/COS/EXP, whose values depend on the math library);
* large wide-encoded tapes agree with recursive evaluation of the
  unsimplified DAG.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import frep
import oracle
from frep import csg, scenes

GOLDEN = np.load(Path(__file__).parent / "golden" / "ref_tapes.npz")
NAMES = [str(n) for n in GOLDEN["names"]]
TRANSCENDENTAL = {1, 2, 9}  # SIN, COS, EXP


def golden(name):
    g = {k.split("/", 1)[1]: GOLDEN[k] for k in GOLDEN.files if k.startswith(name + "/")}
    return g


@pytest.mark.parametrize("name", NAMES)
def test_compiler_matches_reference_golden(name):
    g = golden(name)
    tape = frep.Tape.from_dag(g["ops"], g["in0"], g["in1"], g["consts"], int(g["root"][0]))
    assert tape.fits_reference
    assert tape.n_slots == int(g["ref_slots"][0])
    np.testing.assert_array_equal(tape.instructions, g["ref_instrs"])
    np.testing.assert_array_equal(tape.constant_pool.view(np.uint32), g["ref_consts"].view(np.uint32))


@pytest.mark.parametrize("name", NAMES)
def test_point_eval_matches_reference_eval(name):
    g = golden(name)
    tape = frep.Tape.from_dag(g["ops"], g["in0"], g["in1"], g["consts"], int(g["root"][0]))
    ops = set(int(w) & 0xFF for w in g["ref_instrs"])
    host = tape.eval_points(g["points"])
    orc = np.array([oracle.eval_point(tape.wide(), tape.n_slots, *p) for p in g["points"]], np.float32)
    np.testing.assert_array_equal(host.view(np.uint32), orc.view(np.uint32))
    if ops & TRANSCENDENTAL:
        # SIN/COS/EXP: the library's own functions vs glibc's; agree to a few ulp per op.
        np.testing.assert_allclose(host, g["ref_eval"], rtol=2e-5, atol=2e-5)
    else:
        np.testing.assert_array_equal(host.view(np.uint32), g["ref_eval"].view(np.uint32))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference bridge not built")
@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("n", [2, 5, 12, 20])
def test_compiler_matches_live_reference_random(n, seed):
    dag = scenes.random_csg(n, seed=100 + seed).shape.flatten()
    ref = oracle.RefTape(*dag)
    mine = frep.Tape.from_dag(*dag)
    assert ref.fits == mine.fits_reference
    if ref.fits:
        np.testing.assert_array_equal(mine.instructions, ref.instrs)
        np.testing.assert_array_equal(mine.constant_pool, ref.consts)
        assert mine.n_slots == ref.n_slots


@pytest.mark.skipif(not oracle.ref_available(), reason="reference bridge not built")
def test_constant_folding_identities_match_reference():
    x, y = csg.X(), csg.Y()
    exprs = [
        (-x) + (-y), -(x - y), x * -1.0, -1.0 * (x + 1.0), (-x) * y, x / 4.0, x / -1.0, 0.0 - x,
        x - (-y), csg.Min(x, x), csg.Max(y, x) + csg.Max(x, y), 0.0 * x + 1.0 * y, (x + 0.0) / 1.0,
        csg.Sqrt(csg.Square(x - 2.0)) - csg.Sqrt(csg.Square(2.0 - x)) + csg.Exp(-(-csg.T())),
    ]
    for e in exprs:
        dag = (e + csg.Z()).flatten()
        ref = oracle.RefTape(*dag)
        mine = frep.Tape.from_dag(*dag)
        np.testing.assert_array_equal(mine.instructions, ref.instrs)
        np.testing.assert_array_equal(mine.constant_pool, ref.consts)


def test_wide_tape_large_scene_evaluates_like_the_dag():
    sc = scenes.random_csg(256, seed=2)
    tape = frep.Tape(sc.shape)
    assert not tape.fits_reference and tape.n_instr > 3000
    rng = np.random.default_rng(0)
    pts = np.concatenate([rng.uniform(-1.2, 1.2, (24, 3)), np.zeros((24, 1))], 1).astype(np.float32)
    got = tape.eval_points(pts)
    want = np.array([sc.shape.eval(*p) for p in pts], np.float32)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6)


def test_compile_errors_are_reported():
    with pytest.raises(frep.FrepError) as e:
        frep.Tape(csg.X())
    assert e.value.status == frep._lib.ERR_COMPILE
    with pytest.raises(frep.FrepError):
        frep.Tape(csg.X() + float("nan"))


def test_reference_tape_import_roundtrip():
    g = golden("spheres_union_16")
    t = frep.Tape.from_reference(g["ref_instrs"], g["ref_consts"])
    assert t.n_instr == len(g["ref_instrs"])
    np.testing.assert_array_equal(t.instructions, g["ref_instrs"])
    u = frep.Tape.from_dag(g["ops"], g["in0"], g["in1"], g["consts"], int(g["root"][0]))
    np.testing.assert_array_equal(t.wide(), u.wide())
    bad = g["ref_instrs"].copy()
    bad[0] = (int(bad[0]) & 0xFFFFFF00) | 0x3F  # unknown opcode
    with pytest.raises(frep.FrepError):
        frep.Tape.from_reference(bad, g["ref_consts"])


def test_wide_import_round_trip():
    """frep_tape_from_wide accepts what frep_tape_get_instrs returns and
    derives the same slot count, MIN/MAX count and time use."""
    from frep import scenes
    for expr in (scenes.random_csg(12, seed=8).shape, scenes.Morph(), scenes.TwistedTower(2)):
        a = frep.Tape(expr)
        b = frep.Tape.from_wide(a.wide())
        np.testing.assert_array_equal(a.wide(), b.wide())
        assert (b.n_slots, b.n_minmax, b.uses_time) == (a.n_slots, a.n_minmax, a.uses_time)
        assert not b.fits_reference
        pts = np.random.default_rng(0).uniform(-2, 2, (64, 4)).astype(np.float32)
        np.testing.assert_array_equal(a.eval_points(pts), b.eval_points(pts))


def test_wide_import_rejects_bad_tapes():
    a = frep.Tape(frep.csg.X() * frep.csg.Y() + 1.0).wide()
    bad_op = a.copy()
    bad_op[0] = (bad_op[0] & ~np.uint64(0xFF)) | np.uint64(13)
    not_slot0 = a[:-1] if len(a) > 1 else a
    with pytest.raises(frep.FrepError):
        frep.Tape.from_wide(bad_op)
    with pytest.raises(frep.FrepError):
        frep.Tape.from_wide(np.zeros(0, np.uint64))
    if len(a) > 1 and ((int(a[-2]) >> 16) & 0xFFFF) != 0:
        with pytest.raises(frep.FrepError):
            frep.Tape.from_wide(not_slot0)


@pytest.mark.parametrize("n,seed", [(64, 3), (256, 2), (700, 9)])
def test_constant_reload_keeps_values_and_cuts_slots(n, seed):
    """Beyond the 8-bit encoding, reloading far-away constants changes only
    CONSTs and slot numbers: the other instructions keep their order and
    opcodes, every point value is bit-identical, and fewer slots are used."""
    expr = scenes.random_csg(n, seed=seed).shape
    plain = frep.Tape(expr, const_reload=0xFFFFFFFF)
    packed = frep.Tape(expr)
    assert not packed.fits_reference
    wp, wk = plain.wide(), packed.wide()
    ops_p, ops_k = wp & np.uint64(0xFF), wk & np.uint64(0xFF)
    np.testing.assert_array_equal(ops_p[ops_p != 0], ops_k[ops_k != 0])
    assert (ops_k == 0).sum() > (ops_p == 0).sum()
    assert packed.n_slots < plain.n_slots
    assert packed.n_minmax == plain.n_minmax and packed.uses_time == plain.uses_time
    pts = np.random.default_rng(seed).uniform(-1.3, 1.3, (4000, 4)).astype(np.float32)
    np.testing.assert_array_equal(plain.eval_points(pts), packed.eval_points(pts))
    # the oracle's interval view agrees too
    for lo, hi in (([-0.4, -0.3, -0.2], [0.1, 0.2, 0.3]), ([0.2, 0.1, -0.9], [0.25, 0.15, -0.85])):
        iv_p, ch_p = oracle.eval_interval(wp, plain.n_slots, lo, hi, 0.0, 1)
        iv_k, ch_k = oracle.eval_interval(wk, packed.n_slots, lo, hi, 0.0, 1)
        np.testing.assert_array_equal(iv_p, iv_k)
        np.testing.assert_array_equal(ch_p, ch_k)


def test_small_tapes_keep_the_reference_stream():
    expr = scenes.spheres_union(16).shape
    a, b = frep.Tape(expr), frep.Tape(expr, const_reload=0xFFFFFFFF)
    assert a.fits_reference
    np.testing.assert_array_equal(a.wide(), b.wide())
