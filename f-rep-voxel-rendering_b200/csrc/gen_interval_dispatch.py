"""Writes interval_dispatch.cuh: the interval interpreter's forward loop as
inline PTX with a jump table (brx.idx), for both roundings (0 nearest, 1
outward) and 2 cells per lane (with one cell per lane, a single tree's root
level, the C++ loop measured faster).

The C++ loop tests opcodes in frequency order (two to four compare-and-branch
pairs per instruction); here one indexed branch dispatches each instruction.
Semantics are those of iv_exec / iv_apply in voxelizer.cu and
device_common.cuh, operation for operation: ADD / SUB with the bounds rounded
down / up (or to nearest), MUL as the minimum / maximum of the four endpoint
products (min_sel / max_sel trees, the same order), MIN / MAX with their
choice ballots stored by lane 0 while mm < mm_cap, NEG, SQRT of the bounds
clamped at 0, COPY, CONST. DIV, SIN, COS and EXP (and any other index) leave
the loop so that the caller runs that instruction in C++ and calls again.

    python gen_interval_dispatch.py   (from this directory; the output is committed)
"""
from pathlib import Path

OPS = {"CONST": 0, "SIN": 1, "COS": 2, "ADD": 3, "SUB": 4, "MUL": 5, "DIV": 6, "MIN": 7, "MAX": 8,
       "EXP": 9, "NEG": 10, "SQRT": 11, "COPY": 12}
INLINE = ["CONST", "ADD", "SUB", "MUL", "MIN", "MAX", "NEG", "SQRT", "COPY"]


def min_sel(d, a, b):
    """d = min_sel(a, b) = (b < a) ? b : a"""
    return [f"setp.lt.f32 %%p, {b}, {a};", f"selp.f32 {d}, {b}, {a}, %%p;"]


def max_sel(d, a, b):
    """d = max_sel(a, b) = (a < b) ? b : a"""
    return [f"setp.lt.f32 %%p, {a}, {b};", f"selp.f32 {d}, {b}, {a}, %%p;"]


def cell_ops(op, rnd, h):
    """PTX for cell h: lo / hi into %%qlh / %%qhh from %%alh, %%ahh, %%blh, %%bhh."""
    al, ah, bl, bh = f"%%al{h}", f"%%ah{h}", f"%%bl{h}", f"%%bh{h}"
    ql, qh = f"%%ql{h}", f"%%qh{h}"
    dn, up = ("rm", "rp") if rnd else ("rn", "rn")
    if op == "ADD":
        return [f"add.{dn}.f32 {ql}, {al}, {bl};", f"add.{up}.f32 {qh}, {ah}, {bh};"]
    if op == "SUB":
        return [f"sub.{dn}.f32 {ql}, {al}, {bh};", f"sub.{up}.f32 {qh}, {ah}, {bl};"]
    if op == "MUL":
        out = []
        if rnd:
            prods = [(al, bl), (al, bh), (ah, bl), (ah, bh)]
            for i, (x, y) in enumerate(prods):
                out.append(f"mul.rm.f32 %%l{i}, {x}, {y};")
            for i, (x, y) in enumerate(prods):
                out.append(f"mul.rp.f32 %%u{i}, {x}, {y};")
        else:
            for i, (x, y) in enumerate([(al, bl), (al, bh), (ah, bl), (ah, bh)]):
                out.append(f"mul.rn.f32 %%l{i}, {x}, {y};")
                out.append(f"mov.f32 %%u{i}, %%l{i};")
        out += min_sel("%%t0", "%%l0", "%%l1") + min_sel("%%t1", "%%l2", "%%l3") + min_sel(ql, "%%t0", "%%t1")
        out += max_sel("%%t0", "%%u0", "%%u1") + max_sel("%%t1", "%%u2", "%%u3") + max_sel(qh, "%%t0", "%%t1")
        return out
    if op in ("MIN", "MAX"):
        sel = min_sel if op == "MIN" else max_sel
        return sel(ql, al, bl) + sel(qh, ah, bh)
    if op == "NEG":
        return [f"neg.f32 {ql}, {ah};", f"neg.f32 {qh}, {al};"]
    if op == "SQRT":
        return (max_sel("%%t0", "0f00000000", al) + max_sel("%%t1", "0f00000000", ah) +
                [f"sqrt.{dn}.f32 {ql}, %%t0;", f"sqrt.{up}.f32 {qh}, %%t1;"])
    if op == "COPY":
        return [f"mov.f32 {ql}, {al};", f"mov.f32 {qh}, {ah};"]
    raise ValueError(op)


def choices(op, h):
    """The choice bits of cell h (iv_exec): first_low = a.hi < b.lo,
    second_low = b.hi < a.lo; MIN: FIRST if first_low, else SECOND if
    second_low, else BOTH; MAX the same with FIRST and SECOND swapped. Bit 0
    (the first operand may be the result) into %%c0_h, bit 1 into %%c1_h."""
    al, ah, bl, bh = f"%%al{h}", f"%%ah{h}", f"%%bl{h}", f"%%bh{h}"
    out = [f"setp.lt.f32 %%pf, {ah}, {bl};", f"setp.lt.f32 %%ps, {bh}, {al};",
           "not.pred %%ps, %%ps;", "or.pred %%ps, %%pf, %%ps;",   # first_low || !second_low
           "not.pred %%pf, %%pf;"]                                 # !first_low
    if op == "MIN":
        out += [f"vote.sync.ballot.b32 %%c0_{h}, %%ps, -1;", f"vote.sync.ballot.b32 %%c1_{h}, %%pf, -1;"]
    else:
        out += [f"vote.sync.ballot.b32 %%c0_{h}, %%pf, -1;", f"vote.sync.ballot.b32 %%c1_{h}, %%ps, -1;"]
    return out


def gen(rnd, KI):
    cells = range(KI)
    lo_hi = lambda p: ", ".join(f"%%{p}l{h}, %%{p}h{h}" for h in cells)
    vec = f".v{2 * KI}"
    lines = ["{",
             ".reg .pred %%p, %%pf, %%ps, %%done, %%lane0, %%st;",
             ".reg .b32 %%j, %%m, %%sb, %%lb, %%ad, %%da, %%x, %%y, %%z, %%w, %%nx, %%ny, %%nz, %%nw, %%mm, %%cap, %%ln;",
             ".reg .b32 " + ", ".join(f"%%c0_{h}, %%c1_{h}" for h in cells) + ";",
             ".reg .b64 %%mb, %%ma, %%mo;",
             ".reg .f32 " + ", ".join([lo_hi("a"), lo_hi("b"), lo_hi("q")]) + ";",
             ".reg .f32 %%l0, %%l1, %%l2, %%l3, %%u0, %%u1, %%u2, %%u3, %%t0, %%t1;",
             # operands: %0 = j, %1 = mm (in/out); %2 sbase, %3 m, %4 lane_base, %5 mmb, %6 mm_cap
             "mov.b32 %%j, %0;", "mov.b32 %%mm, %1;", "mov.b32 %%sb, %2;", "mov.b32 %%m, %3;",
             "mov.b32 %%lb, %4;", "mov.b64 %%mb, %5;", "mov.b32 %%cap, %6;",
             "mov.u32 %%ln, %%laneid;", "setp.eq.u32 %%lane0, %%ln, 0;",
             # decode word j, then each iteration loads word j + 1 before
             # dispatching j (word m, one past the chunk, is in the staging area)
             "mad.lo.u32 %%da, %%j, 16, %%sb;",
             "ld.shared.v4.u32 {%%x, %%y, %%z, %%w}, [%%da];",
             "$FRI_LOOP:",
             "setp.ge.u32 %%done, %%j, %%m;",
             "@%%done bra.uni $FRI_EXIT;",
             "ld.shared.v4.u32 {%%nx, %%ny, %%nz, %%nw}, [%%da+16];",
             "and.b32 %%x, %%x, 15;"]
    names = {v: n for n, v in OPS.items()}
    targets = [f"$FRI_{names[i]}" if names.get(i) in INLINE else "$FRI_EXIT" for i in range(16)]
    lines.append("$FRI_TAB: .branchtargets " + ", ".join(targets) + ";")
    lines.append("brx.idx.uni %%x, $FRI_TAB;")
    lines.append("$FRI_CONST:")
    for h in cells:
        lines += [f"mov.b32 %%ql{h}, %%y;", f"mov.b32 %%qh{h}, %%y;"]
    lines.append("bra.uni $FRI_STORE;")
    ld_a = ["add.u32 %%ad, %%lb, %%y;", f"ld.shared{vec}.f32 {{{lo_hi('a')}}}, [%%ad];"]
    ld_b = ["add.u32 %%ad, %%lb, %%z;", f"ld.shared{vec}.f32 {{{lo_hi('b')}}}, [%%ad];"]
    for op in ["ADD", "SUB", "MUL", "MIN", "MAX", "NEG", "SQRT", "COPY"]:
        binary = op in ("ADD", "SUB", "MUL", "MIN", "MAX")
        lines.append(f"$FRI_{op}:")
        lines += ld_a + (ld_b if binary else [])
        for h in cells:
            lines += cell_ops(op, rnd, h)
        if op in ("MIN", "MAX"):
            for h in cells:
                lines += choices(op, h)
            # lane 0 records the ballots while mm < mm_cap; mm counts every MIN / MAX
            lines += ["setp.lt.and.u32 %%st, %%mm, %%cap, %%lane0;",
                      f"mul.wide.u32 %%mo, %%mm, {8 * KI};", "add.s64 %%ma, %%mb, %%mo;"]
            if KI == 1:
                lines.append("@%%st st.global.v2.u32 [%%ma], {%%c0_0, %%c1_0};")
            else:
                lines.append("@%%st st.global.v4.u32 [%%ma], {%%c0_0, %%c1_0, %%c0_1, %%c1_1};")
            lines.append("add.u32 %%mm, %%mm, 1;")
        lines.append("bra.uni $FRI_STORE;")
    lines += ["$FRI_STORE:",
              "add.u32 %%ad, %%lb, %%w;",
              f"st.shared{vec}.f32 [%%ad], {{{lo_hi('q')}}};",
              "add.u32 %%j, %%j, 1;",
              "add.u32 %%da, %%da, 16;",
              "mov.b32 %%x, %%nx;", "mov.b32 %%y, %%ny;", "mov.b32 %%z, %%nz;", "mov.b32 %%w, %%nw;",
              "bra.uni $FRI_LOOP;",
              "$FRI_EXIT:",
              "mov.b32 %0, %%j;",
              "mov.b32 %1, %%mm;",
              "}"]
    return lines


def emit(rnd, KI):
    asm = "\n".join(f'        "{l}\\n\\t"' for l in gen(rnd, KI))
    return f'''// Runs decoded instructions j .. m-1 of the staged chunk at shared address
// sbase on {KI} cell(s) per lane ({"outward" if rnd else "nearest"} rounding; slot rows at lane_base),
// recording MIN / MAX choices at mmb[mm] (mm counted on). Returns at m, or at
// the first instruction the loop does not run (DIV, SIN, COS, EXP).
__device__ __noinline__ IvRun iv_run_{rnd}_{KI}(uint32_t sbase, uint32_t j, uint32_t m, uint32_t lane_base,
                                       uint2* mmb, uint32_t mm, uint32_t mm_cap) {{
    asm volatile(
{asm}
        : "+r"(j), "+r"(mm)
        : "r"(sbase), "r"(m), "r"(lane_base), "l"(mmb), "r"(mm_cap)
        : "memory");
    return IvRun{{j, mm}};
}}
'''


def text() -> str:
    """The header's contents."""
    head = '''// Generated by gen_interval_dispatch.py: the interval interpreter's forward
// loop with a jump table (brx.idx). Included by voxelizer.cu.
#pragma once

struct IvRun {
    uint32_t j, mm;
};

'''
    return head + "\n".join(emit(r, 2) for r in (0, 1))


def main():
    out = Path(__file__).with_name("interval_dispatch.cuh")
    out.write_text(text())
    print("wrote", out)


if __name__ == "__main__":
    main()
