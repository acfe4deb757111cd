"""Writes point_dispatch.cuh: the point interpreter's inner loop as inline PTX
with a jump table (brx.idx), for 2, 4 and 8 cells per lane (8: a slot row is
two 16-byte halves 512 bytes apart, as lds_k / sts_k lay it out).

The loop in C++ is a switch over (opcode, forward-A, forward-B); the compiler
lowers it to a tree of compares and branches (about six per tape instruction).
Here one indexed branch dispatches each instruction. Semantics are those of
pt_exec in voxelizer.cu, operation for operation (round-to-nearest add / sub /
mul / div / sqrt, min_sel / max_sel as compare + select, neg, copy, const);
SIN, COS and EXP, and any other index, leave the loop so that the caller runs
that instruction in C++ and calls again.

    python gen_point_dispatch.py   (from this directory; the output is committed)
"""
from pathlib import Path

OPS = {"CONST": 0, "SIN": 1, "COS": 2, "ADD": 3, "SUB": 4, "MUL": 5, "DIV": 6, "MIN": 7, "MAX": 8,
       "EXP": 9, "NEG": 10, "SQRT": 11, "COPY": 12}
FA, FB = 16, 32
BINARY = ["ADD", "SUB", "MUL", "DIV", "MIN", "MAX"]
UNARY = ["NEG", "SQRT", "COPY"]


def body(op, k, a, b):
    """PTX computing q<k> = op(a, b) (a, b: register names)."""
    q = f"%%q{k}"
    if op == "ADD":
        return [f"add.rn.f32 {q}, {a}, {b};"]
    if op == "SUB":
        return [f"sub.rn.f32 {q}, {a}, {b};"]
    if op == "MUL":
        return [f"mul.rn.f32 {q}, {a}, {b};"]
    if op == "DIV":
        return [f"div.rn.f32 {q}, {a}, {b};"]
    if op == "MIN":  # min_sel: (b < a) ? b : a
        return [f"setp.lt.f32 %%p, {b}, {a};", f"selp.f32 {q}, {b}, {a}, %%p;"]
    if op == "MAX":  # max_sel: (a < b) ? b : a
        return [f"setp.lt.f32 %%p, {a}, {b};", f"selp.f32 {q}, {b}, {a}, %%p;"]
    if op == "NEG":
        return [f"neg.f32 {q}, {a};"]
    if op == "SQRT":
        return [f"sqrt.rn.f32 {q}, {a};"]
    if op == "COPY":
        return [f"mov.f32 {q}, {a};"]
    raise ValueError(op)


K8_HALF = 32 * 16  # bytes between the two halves of an 8-cell slot row


def gen(K):
    regs = lambda p: ", ".join(f"%%{p}{i}" for i in range(K))

    def half(p, h):
        return ", ".join(f"%%{p}{i}" for i in range(4 * h, 4 * h + 4))

    def ld(p, off):
        if K == 8:
            return [f"add.u32 %%ad, %%lb, {off};", f"ld.shared.v4.f32 {{{half(p, 0)}}}, [%%ad];",
                    f"ld.shared.v4.f32 {{{half(p, 1)}}}, [%%ad+{K8_HALF}];"]
        return [f"add.u32 %%ad, %%lb, {off};", f"ld.shared.v{K}.f32 {{{regs(p)}}}, [%%ad];"]
    lines = []
    lines.append("{")
    lines.append(".reg .pred %%p, %%done;")
    lines.append(".reg .b32 %%j, %%m, %%sb, %%lb, %%ad, %%da, %%x, %%y, %%z, %%w, %%nx, %%ny, %%nz, %%nw;")
    lines.append(f".reg .f32 {regs('q')}, {regs('a')}, {regs('b')};")
    # operands: %0 = j (in/out), %1..%K = r (in/out), then sbase, m, lane_base
    lines.append("mov.b32 %%j, %0;")
    for i in range(K):
        lines.append(f"mov.f32 %%q{i}, %{1 + i};")
    lines.append(f"mov.b32 %%sb, %{K + 1};")
    lines.append(f"mov.b32 %%m, %{K + 2};")
    lines.append(f"mov.b32 %%lb, %{K + 3};")
    # decode word j, then each iteration loads word j + 1 before dispatching j
    # (word m, one past the chunk, is in the staging area: it holds STAGE + 1)
    lines.append("mad.lo.u32 %%da, %%j, 16, %%sb;")
    lines.append("ld.shared.v4.u32 {%%x, %%y, %%z, %%w}, [%%da];")
    lines.append("$FRP_LOOP:")
    lines.append("setp.ge.u32 %%done, %%j, %%m;")
    lines.append("@%%done bra.uni $FRP_EXIT;")
    lines.append("ld.shared.v4.u32 {%%nx, %%ny, %%nz, %%nw}, [%%da+16];")
    lines.append("and.b32 %%x, %%x, 63;")
    targets = []
    for idx in range(64):
        op, fa, fb = idx & 15, bool(idx & FA), bool(idx & FB)
        name = next((n for n, v in OPS.items() if v == op), None)
        if name == "CONST" and not fa and not fb:
            targets.append("$FRP_CONST")
        elif name in BINARY:
            targets.append(f"$FRP_{name}_{int(fa)}{int(fb)}")
        elif name in UNARY and not fb:
            targets.append(f"$FRP_{name}_{int(fa)}0")
        else:
            targets.append("$FRP_EXIT")
    lines.append("$FRP_TAB: .branchtargets " + ", ".join(targets) + ";")
    lines.append("brx.idx.uni %%x, $FRP_TAB;")

    # Each case ends with the store of its result and the dispatch of the next
    # instruction (a threaded loop: no jump back to a common loop head).
    def store_next():
        out = ["add.u32 %%ad, %%lb, %%w;"]
        if K == 8:
            out.append(f"st.shared.v4.f32 [%%ad], {{{half('q', 0)}}};")
            out.append(f"st.shared.v4.f32 [%%ad+{K8_HALF}], {{{half('q', 1)}}};")
        else:
            out.append(f"st.shared.v{K}.f32 [%%ad], {{{regs('q')}}};")
        out += ["add.u32 %%j, %%j, 1;", "add.u32 %%da, %%da, 16;",
                "mov.b32 %%x, %%nx;", "mov.b32 %%y, %%ny;", "mov.b32 %%z, %%nz;", "mov.b32 %%w, %%nw;",
                "setp.ge.u32 %%done, %%j, %%m;", "@%%done bra.uni $FRP_EXIT;",
                "ld.shared.v4.u32 {%%nx, %%ny, %%nz, %%nw}, [%%da+16];",
                "and.b32 %%x, %%x, 63;", "brx.idx.uni %%x, $FRP_TAB;"]
        return out
    # CONST: the value's bits are the decode word's y
    lines.append("$FRP_CONST:")
    for i in range(K):
        lines.append(f"mov.b32 %%q{i}, %%y;")
    lines += store_next()
    for name in BINARY:
        for fa in (0, 1):
            for fb in (0, 1):
                lines.append(f"$FRP_{name}_{fa}{fb}:")
                if not fa:
                    lines += ld("a", "%%y")
                if not fb:
                    lines += ld("b", "%%z")
                for i in range(K):
                    lines += body(name, i, f"%%q{i}" if fa else f"%%a{i}", f"%%q{i}" if fb else f"%%b{i}")
                lines += store_next()
    for name in UNARY:
        for fa in (0, 1):
            lines.append(f"$FRP_{name}_{fa}0:")
            if not fa:
                lines += ld("a", "%%y")
            for i in range(K):
                lines += body(name, i, f"%%q{i}" if fa else f"%%a{i}", None)
            lines += store_next()
    lines.append("$FRP_EXIT:")
    lines.append("mov.b32 %0, %%j;")
    for i in range(K):
        lines.append(f"mov.f32 %{1 + i}, %%q{i};")
    lines.append("}")
    return lines


def emit(K):
    outs = ", ".join(['"+r"(j)'] + [f'"+f"(r.v[{i}])' for i in range(K)])
    ins = '"r"(sbase), "r"(m), "r"(lane_base)'
    asm = "\n".join(f'        "{l}\\n\\t"' for l in gen(K))
    return f'''// Runs decoded instructions j .. m-1 of the staged chunk at shared address
// sbase on {K} cells per lane (slot rows at lane_base), the running result in r.
// Returns at m, or at the first instruction the loop does not run (SIN, COS,
// EXP): its index, with r the previous instruction's result.
__device__ __noinline__ PtRun<{K}> pt_run_{K}(uint32_t sbase, uint32_t j, uint32_t m, uint32_t lane_base,
                                          FK<{K}> r) {{
    asm volatile(
{asm}
        : {outs}
        : {ins}
        : "memory");
    return PtRun<{K}>{{j, r}};
}}
'''


def text() -> str:
    """The header's contents."""
    head = '''// Generated by gen_point_dispatch.py: the point interpreter's inner loop with
// a jump table (brx.idx). Included by voxelizer.cu after FK<K> is defined.
#pragma once

template <int K>
struct PtRun {
    uint32_t j;
    FK<K> r;
};

'''
    return head + emit(2) + "\n" + emit(4) + "\n" + emit(8)


def main():
    out = Path(__file__).with_name("point_dispatch.cuh")
    out.write_text(text())
    print("wrote", out)


if __name__ == "__main__":
    main()
