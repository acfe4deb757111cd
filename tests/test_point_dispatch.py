"""The point interpreter's jump-table loop (csrc/point_dispatch.cuh) is the
output of its generator (csrc/gen_point_dispatch.py), and the generator's
case table covers every (opcode, forwarding) index the decoder can produce:
CONST, the six binary operations with each forwarding pair, NEG / SQRT /
COPY with or without a forwarded operand; SIN / COS / EXP and every other
index leave the loop for the C++ switch."""
from __future__ import annotations

import importlib.util
from pathlib import Path

CSRC = Path(__file__).resolve().parents[1] / "f-rep-voxel-rendering_b200" / "csrc"


def _gen():
    spec = importlib.util.spec_from_file_location("gen_point_dispatch", CSRC / "gen_point_dispatch.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_header_is_the_generator_output():
    assert (CSRC / "point_dispatch.cuh").read_text() == _gen().text()


def test_case_table():
    g = _gen()
    for k in (2, 4, 8):
        lines = g.gen(k)
        tab = next(l for l in lines if ".branchtargets" in l)
        targets = tab.split(".branchtargets", 1)[1].strip(" ;").split(", ")
        assert len(targets) == 64
        for idx, t in enumerate(targets):
            op, fa, fb = idx & 15, idx >> 4 & 1, idx >> 5 & 1
            name = {v: n for n, v in g.OPS.items()}.get(op)
            if name == "CONST" and not fa and not fb:
                assert t == "$FRP_CONST"
            elif name in g.BINARY:
                assert t == f"$FRP_{name}_{fa}{fb}"
            elif name in g.UNARY and not fb:
                assert t == f"$FRP_{name}_{fa}0"
            else:
                assert t == "$FRP_EXIT", (idx, t)
        # every target is defined once
        for t in set(targets):
            assert sum(1 for l in lines if l == t + ":") == 1, t


def test_interval_header_is_the_generator_output():
    spec = importlib.util.spec_from_file_location("gen_interval_dispatch", CSRC / "gen_interval_dispatch.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert (CSRC / "interval_dispatch.cuh").read_text() == mod.text()
    for rnd in (0, 1):
        lines = mod.gen(rnd, 2)
        tab = next(l for l in lines if ".branchtargets" in l)
        targets = tab.split(".branchtargets", 1)[1].strip(" ;").split(", ")
        assert len(targets) == 16
        inline = {mod.OPS[n] for n in mod.INLINE}
        for idx, t in enumerate(targets):
            assert (t != "$FRI_EXIT") == (idx in inline), (idx, t)
        for t in set(targets):
            assert sum(1 for l in lines if l == t + ":") == 1, t
