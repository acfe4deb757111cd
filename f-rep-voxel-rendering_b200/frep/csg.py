"""Scene construction API: expression DAG and primitive library.

Mirrors the reference's ``csg`` namespace so that scene code reads the same:

* ``Operator`` and ``Expr`` follow ``vulkan/include/csg/expression.h:14-118``
  (operator numbering, arithmetic operators, ``X/Y/Z/T``, ``Sin`` .. ``Sqrt``,
  and substitution ``e(newX, newY, newZ, newT)`` = ``expression.cpp:281-295``).
* ``Vector3`` and the shape functions follow ``vulkan/include/csg/lib.h:8-67`` /
  ``vulkan/src/csg/lib.cpp:1-216`` (``Sphere`` is squared distance minus squared
  radius, ``Box`` a max of squared slabs, ``Abs`` = ``Sqrt(x*x)``, transforms by
  substitution).

Constants are held as float32, exactly as the reference's ``Expr(float)``
constructor stores them. An expression is turned into a flat DAG
(``Expr.flatten()``) that crosses the C-ABI (``frep_dag`` in ``include/frep.h``).
"""
from __future__ import annotations

from enum import IntEnum

import numpy as np


class Operator(IntEnum):
    """csg::Operator (vulkan/include/csg/expression.h:14-22)."""

    X = 0
    Y = 1
    Z = 2
    T = 3
    CONST = 4
    SIN = 5
    COS = 6
    EXP = 7
    NEG = 8
    SQRT = 9
    ADD = 10
    SUB = 11
    MUL = 12
    DIV = 13
    MIN = 14
    MAX = 15


ARITY = (0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2)
_AXES = (Operator.X, Operator.Y, Operator.Z, Operator.T)


def f32(x) -> float:
    """Rounds a Python number to float32, as C++ does when building Expr(float)."""
    return float(np.float32(x))


class Node:
    """One DAG node: an operator, its input expressions and (for CONST) a value."""

    __slots__ = ("op", "inputs", "constant")

    def __init__(self, op: Operator, inputs=(), constant: float = 0.0):
        self.op = Operator(op)
        self.inputs = tuple(inputs)
        self.constant = constant


class Expr:
    """A handle on a DAG node, passed by value like the reference's csg::Expr."""

    __slots__ = ("node",)

    def __init__(self, value=None):
        if value is None:
            self.node = None
        elif isinstance(value, Node):
            self.node = value
        elif isinstance(value, Expr):
            self.node = value.node
        else:
            self.node = Node(Operator.CONST, (), f32(value))

    # -- predicates (expression.cpp:21-62) ---------------------------------
    def is_axis_op(self) -> bool:
        return self.node.op in _AXES

    def is_constant_op(self, value=None) -> bool:
        if self.node.op != Operator.CONST:
            return False
        return value is None or self.node.constant == f32(value)

    def is_input_op(self) -> bool:
        return self.node.op >= Operator.SIN

    def is_op(self, op: Operator) -> bool:
        return self.node.op == op

    def __getitem__(self, i: int) -> "Expr":
        return self.node.inputs[i]

    # -- arithmetic (expression.cpp:79-105) --------------------------------
    def __neg__(self):
        return _make(Operator.NEG, self)

    def __add__(self, o):
        return _make(Operator.ADD, self, _wrap(o))

    def __radd__(self, o):
        return _make(Operator.ADD, _wrap(o), self)

    def __sub__(self, o):
        return _make(Operator.SUB, self, _wrap(o))

    def __rsub__(self, o):
        return _make(Operator.SUB, _wrap(o), self)

    def __mul__(self, o):
        return _make(Operator.MUL, self, _wrap(o))

    def __rmul__(self, o):
        return _make(Operator.MUL, _wrap(o), self)

    def __truediv__(self, o):
        return _make(Operator.DIV, self, _wrap(o))

    def __rtruediv__(self, o):
        return _make(Operator.DIV, _wrap(o), self)

    # -- traversal ------------------------------------------------------------
    def topo(self):
        """Nodes in csg::Expr::TopoIter order: depth-first, inputs in order,
        a node after all its inputs, each node once (expression.cpp:298-314)."""
        order, seen = [], set()
        stack = [(self.node, False)]
        while stack:
            node, expanded = stack.pop()
            if expanded:
                order.append(node)
                continue
            if id(node) in seen:
                continue
            seen.add(id(node))
            stack.append((node, True))
            for child in reversed(node.inputs):
                if id(child.node) not in seen:
                    stack.append((child.node, False))
        return order

    def node_count(self) -> int:
        return len(self.topo())

    def __call__(self, new_x, new_y, new_z, new_t) -> "Expr":
        """Substitutes the axes (expression.cpp:281-295): every operator node is
        rebuilt, constants are kept, X/Y/Z/T are replaced."""
        repl = {Operator.X: _wrap(new_x), Operator.Y: _wrap(new_y),
                Operator.Z: _wrap(new_z), Operator.T: _wrap(new_t)}
        mapped = {}
        for node in self.topo():
            if node.op in repl:
                mapped[id(node)] = repl[node.op]
            elif node.op == Operator.CONST:
                mapped[id(node)] = Expr(node)
            else:
                mapped[id(node)] = Expr(Node(node.op, [mapped[id(c.node)] for c in node.inputs]))
        return mapped[id(self.node)]

    def flatten(self):
        """Flat DAG arrays (ops u8, in0 u32, in1 u32, consts f32, root) in
        topological order; node identity is preserved."""
        order = self.topo()
        index = {id(n): i for i, n in enumerate(order)}
        n = len(order)
        ops = np.zeros(n, np.uint8)
        in0 = np.zeros(n, np.uint32)
        in1 = np.zeros(n, np.uint32)
        consts = np.zeros(n, np.float32)
        for i, node in enumerate(order):
            ops[i] = int(node.op)
            if node.inputs:
                in0[i] = index[id(node.inputs[0].node)]
                if len(node.inputs) > 1:
                    in1[i] = index[id(node.inputs[1].node)]
            if node.op == Operator.CONST:
                consts[i] = node.constant
        return ops, in0, in1, consts, index[id(self.node)]

    def eval(self, x, y, z, t=0.0) -> float:
        """Recursive float32 evaluation of the unsimplified DAG (expression.cpp:151-166),
        with glm's min/max selection rules."""
        vals = {}
        xyzt = (np.float32(x), np.float32(y), np.float32(z), np.float32(t))
        with np.errstate(all="ignore"):
            for node in self.topo():
                if node.op in _AXES:
                    v = xyzt[int(node.op)]
                elif node.op == Operator.CONST:
                    v = np.float32(node.constant)
                else:
                    a = vals[id(node.inputs[0].node)]
                    b = vals[id(node.inputs[1].node)] if len(node.inputs) > 1 else None
                    v = _apply(node.op, a, b)
                vals[id(node)] = v
        return float(vals[id(self.node)])


def _apply(op, a, b):
    f = np.float32
    if op == Operator.SIN:
        return f(np.sin(a))
    if op == Operator.COS:
        return f(np.cos(a))
    if op == Operator.EXP:
        return f(np.exp(a))
    if op == Operator.NEG:
        return f(-a)
    if op == Operator.SQRT:
        return f(np.sqrt(a))
    if op == Operator.ADD:
        return f(a + b)
    if op == Operator.SUB:
        return f(a - b)
    if op == Operator.MUL:
        return f(a * b)
    if op == Operator.DIV:
        return f(a / b)
    if op == Operator.MIN:
        return b if b < a else a
    if op == Operator.MAX:
        return b if a < b else a
    raise ValueError(op)


def _wrap(v) -> Expr:
    return v if isinstance(v, Expr) else Expr(v)


def _make(op: Operator, *inputs: Expr) -> Expr:
    return Expr(Node(op, [_wrap(i) for i in inputs]))


# -- leaf and unary builders (expression.cpp:228-278) ------------------------
def X() -> Expr:
    return Expr(Node(Operator.X))


def Y() -> Expr:
    return Expr(Node(Operator.Y))


def Z() -> Expr:
    return Expr(Node(Operator.Z))


def T() -> Expr:
    return Expr(Node(Operator.T))


def Constant(x) -> Expr:
    return Expr(x)


def Sin(e) -> Expr:
    return _make(Operator.SIN, e)


def Cos(e) -> Expr:
    return _make(Operator.COS, e)


def Exp(e) -> Expr:
    return _make(Operator.EXP, e)


def Sqrt(e) -> Expr:
    return _make(Operator.SQRT, e)


def Min(a, b) -> Expr:
    return _make(Operator.MIN, a, b)


def Max(a, b) -> Expr:
    return _make(Operator.MAX, a, b)


# -- lib.h ---------------------------------------------------------------------
class Vector3:
    """Component-wise vector of expressions (lib.h:8-25)."""

    __slots__ = ("x", "y", "z")

    def __init__(self, x, y, z):
        self.x, self.y, self.z = _wrap(x), _wrap(y), _wrap(z)

    def __add__(self, o):
        return Vector3(self.x + o.x, self.y + o.y, self.z + o.z)

    def __sub__(self, o):
        return Vector3(self.x - o.x, self.y - o.y, self.z - o.z)

    def __neg__(self):
        return Vector3(-self.x, -self.y, -self.z)

    def __mul__(self, o):
        if isinstance(o, Vector3):
            return Vector3(self.x * o.x, self.y * o.y, self.z * o.z)
        o = _wrap(o)
        return Vector3(self.x * o, self.y * o, self.z * o)

    def __rmul__(self, o):
        o = _wrap(o)
        return Vector3(o * self.x, o * self.y, o * self.z)

    def __truediv__(self, o):
        if isinstance(o, Vector3):
            return Vector3(self.x / o.x, self.y / o.y, self.z / o.z)
        o = _wrap(o)
        return Vector3(self.x / o, self.y / o, self.z / o)


def _vec(v) -> Vector3:
    return v if isinstance(v, Vector3) else Vector3(*v)


def Empty() -> Expr:
    return Expr(1)


def Axes() -> Vector3:
    return Vector3(X(), Y(), Z())


def Pi() -> Expr:
    return Expr(np.float32(np.pi))


def Square(x) -> Expr:
    x = _wrap(x)
    return x * x


def Abs(x) -> Expr:
    return Sqrt(Square(x))


def Pow(x, p: int) -> Expr:
    x = _wrap(x)
    if p == 0:
        return Constant(1.0)
    if p == 1:
        return x
    if p % 2 == 0:
        return Square(Pow(x, p // 2))
    return Square(Pow(x, p // 2)) * x


def Dot(a, b) -> Expr:
    a, b = _vec(a), _vec(b)
    return a.x * b.x + a.y * b.y + a.z * b.z


def Norm(a) -> Expr:
    a = _vec(a)
    return Sqrt(a.x * a.x + a.y * a.y + a.z * a.z)


def Norm2(a) -> Expr:
    a = _vec(a)
    return a.x * a.x + a.y * a.y + a.z * a.z


def Dist(a, b) -> Expr:
    return Norm(_vec(b) - _vec(a))


def Dist2(a, b) -> Expr:
    return Norm2(_vec(b) - _vec(a))


def Union(a, b) -> Expr:
    return Min(a, b)


def Intersect(a, b) -> Expr:
    return Max(a, b)


def Complement(a) -> Expr:
    return -_wrap(a)


def Diff(a, b) -> Expr:
    return Intersect(a, Complement(b))


def Sphere(center, radius) -> Expr:
    return Dist2(Axes(), _vec(center)) - Square(radius)


def Box(low_vertex, size) -> Expr:
    lo, sz = _vec(low_vertex), _vec(size)
    a = Square(X() - (lo.x + sz.x / 2)) - Square(sz.x / 2)
    b = Square(Y() - (lo.y + sz.y / 2)) - Square(sz.y / 2)
    c = Square(Z() - (lo.z + sz.z / 2)) - Square(sz.z / 2)
    return Intersect(a, Intersect(b, c))


def TranslateX(a, dx) -> Expr:
    return a(X() - dx, Y(), Z(), T())


def TranslateY(a, dy) -> Expr:
    return a(X(), Y() - dy, Z(), T())


def TranslateZ(a, dz) -> Expr:
    return a(X(), Y(), Z() - dz, T())


def TranslateXYZ(a, da) -> Expr:
    da = _vec(da)
    return a(X() - da.x, Y() - da.y, Z() - da.z, T())


def ScaleX(a, s) -> Expr:
    return a(X() / s, Y(), Z(), T())


def ScaleY(a, s) -> Expr:
    return a(X(), Y() / s, Z(), T())


def ScaleZ(a, s) -> Expr:
    return a(X(), Y(), Z() / s, T())


def ScaleXYZ(a, s) -> Expr:
    if isinstance(s, (Vector3, tuple, list)):
        s = _vec(s)
        return a(X() / s.x, Y() / s.y, Z() / s.z, T())
    return a(X() / s, Y() / s, Z() / s, T())


def RotateX(a, angle) -> Expr:
    c = Cos(-_wrap(angle))
    s = Sin(-_wrap(angle))
    return a(X(), c * Y() - s * Z(), s * Y() + c * Z(), T())


def RotateY(a, angle) -> Expr:
    c = Cos(-_wrap(angle))
    s = Sin(-_wrap(angle))
    return a(c * X() + s * Z(), Y(), -s * X() + c * Z(), T())


def RotateZ(a, angle) -> Expr:
    c = Cos(-_wrap(angle))
    s = Sin(-_wrap(angle))
    return a(c * X() - s * Y(), s * X() + c * Y(), Z(), T())
