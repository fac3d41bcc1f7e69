#!/usr/bin/env python3
"""Generator for the straight-line DFT codelets used by the DFTTest kernels.

The codelets are emitted as ``__device__ __forceinline__`` CUDA functions that
operate on register arrays.  Everything here is written from the DFT
definition; no third-party generator output is used.

Building blocks
---------------
* values carry a *lazy constant coefficient*: a value is ``coef * node``.
  Multiplying by a constant is free (it only changes ``coef``); adding two
  values with different coefficients costs exactly one FFMA
  (``a*x + b*y = b*((a/b)*x + y)``).  This automatically yields the
  "tangent" form of twiddle butterflies (6 instructions for ``e +- w*o``).
* hash-consing with sign normalisation gives common-subexpression
  elimination, so the Hermitian redundancy of real-input transforms is
  shared instead of recomputed.
* a dead-code pass keeps only what the requested outputs need.

Transforms (unnormalised, forward sign -1, inverse sign +1, the same
conventions as the reference's kernels, cpu_source/kernel.hpp:19-1721):

* ``r2c_N``   real N-point forward DFT, packed output
  ``[X0.re, X(N/2).re, X1.re, X1.im, ..., X(N/2-1).re, X(N/2-1).im]``
* ``c2r_N``   inverse of the packed layout (imag of bins 0 and N/2 ignored)
* ``cdft_N_fwd`` / ``cdft_N_inv`` complex in-place DFTs (separate re/im arrays)
* ``rdftT_N`` real N-point (N odd) forward DFT, bins 0..N/2 (``im[0]`` = 0)

Run ``python gen_codelets.py`` to rewrite ``codelets.cuh``;
``python gen_codelets.py --check`` evaluates the emitted code in float64
against numpy and prints instruction counts.
"""
from __future__ import annotations

import cmath
import math
import os
import re
import sys

import numpy as np


_FULL_PRECISION = False


def _f32(c: float) -> str:
    if _FULL_PRECISION:
        return repr(float(c)) + "f"
    s = format(float(np.float32(c)), ".9g")
    if "e" not in s and "." not in s:
        s += ".0"
    return s + "f"


class Node:
    __slots__ = ("name", "op", "args", "const")

    def __init__(self, name, op, args=(), const=None):
        self.name = name
        self.op = op  # 'in', 'add', 'sub', 'fma', 'mul'
        self.args = args
        self.const = const


class V:
    """A lazily scaled value: coef * node (node None means exact zero)."""

    __slots__ = ("node", "coef")

    def __init__(self, node, coef=1.0):
        self.node = node
        self.coef = coef if node is not None else 0.0

    @property
    def zero(self):
        return self.node is None or self.coef == 0.0


ZERO = V(None, 0.0)


def _close(a, b):
    return abs(a - b) <= 1e-15 * max(1.0, abs(a), abs(b))


class Gen:
    def __init__(self):
        self.nodes: list[Node] = []
        self.cse: dict = {}
        self.counter = 0

    # -- node creation -------------------------------------------------
    def _node(self, op, args, const=None):
        key = (op, tuple(a.name for a in args), None if const is None else round(const, 15))
        hit = self.cse.get(key)
        if hit is not None:
            return hit
        n = Node(f"t{self.counter}", op, args, const)
        self.counter += 1
        self.nodes.append(n)
        self.cse[key] = n
        return n

    def inp(self, expr):
        n = Node(expr, "in")
        return V(n, 1.0)

    # -- arithmetic on lazy values ---------------------------------------
    def scale(self, x: V, c: float) -> V:
        if x.zero or c == 0.0:
            return ZERO
        return V(x.node, x.coef * c)

    def neg(self, x: V) -> V:
        return self.scale(x, -1.0)

    def add(self, x: V, y: V) -> V:
        if x.zero:
            return y
        if y.zero:
            return x
        if x.node is y.node:
            c = x.coef + y.coef
            return ZERO if abs(c) < 1e-15 else V(x.node, c)
        a, b = x.coef, y.coef
        if _close(abs(a), abs(b)):
            # a*(X +- Y)
            if _close(a, b):
                n1, n2 = sorted((x.node, y.node), key=lambda n: n.name)
                return V(self._node("add", (n1, n2)), a)
            # a*(X - Y) with b = -a
            if x.node.name < y.node.name:
                return V(self._node("sub", (x.node, y.node)), a)
            return V(self._node("sub", (y.node, x.node)), b)
        # a*X + b*Y: keep the coefficient that is +-1 (or the larger one)
        # outside, fold the ratio into an FFMA.
        def keep_outer(c):
            return _close(abs(c), 1.0)

        if keep_outer(b) or (not keep_outer(a) and abs(b) >= abs(a)):
            k = a / b
            return V(self._node("fma", (x.node, y.node), k), b)
        k = b / a
        return V(self._node("fma", (y.node, x.node), k), a)

    def sub(self, x: V, y: V) -> V:
        return self.add(x, self.neg(y))

    # complex helpers: tuples (re, im)
    def cadd(self, x, y):
        return (self.add(x[0], y[0]), self.add(x[1], y[1]))

    def csub(self, x, y):
        return (self.sub(x[0], y[0]), self.sub(x[1], y[1]))

    def cconj(self, x):
        return (x[0], self.neg(x[1]))

    def cmulc(self, x, w: complex):
        """x * w for a constant w (two lazy FFMAs at most)."""
        c, s = w.real, w.imag
        if abs(s) < 1e-15:
            return (self.scale(x[0], c), self.scale(x[1], c))
        if abs(c) < 1e-15:
            return (self.scale(x[1], -s), self.scale(x[0], s))
        re = self.add(self.scale(x[0], c), self.scale(x[1], -s))
        im = self.add(self.scale(x[0], s), self.scale(x[1], c))
        return (re, im)

    # -- materialisation ---------------------------------------------------
    def expr(self, x: V) -> str:
        if x.zero:
            return "0.0f"
        name = x.node.name
        if _close(x.coef, 1.0):
            return name
        if _close(x.coef, -1.0):
            return f"(-{name})"
        return f"({_f32(x.coef)} * {name})"


# ---------------------------------------------------------------------------
# transform algorithms
# ---------------------------------------------------------------------------

def _w(sign, k, n):
    return cmath.exp(sign * 2j * math.pi * k / n)


def cdft(g: Gen, x, sign):
    """Complex DFT of the list of complex lazy values x (any supported n)."""
    n = len(x)
    if n == 1:
        return list(x)
    if n % 2 == 0:
        E = cdft(g, x[0::2], sign)
        O = cdft(g, x[1::2], sign)
        m = n // 2
        out = [None] * n
        for k in range(m):
            t = g.cmulc(O[k], _w(sign, k, n))
            out[k] = g.cadd(E[k], t)
            out[k + m] = g.csub(E[k], t)
        return out
    return odd_dft(g, x, sign)


def odd_dft(g: Gen, x, sign):
    """Odd-length DFT by symmetric/antisymmetric input pairs."""
    n = len(x)
    h = n // 2
    s = [g.cadd(x[j], x[n - j]) for j in range(1, h + 1)]
    d = [g.csub(x[j], x[n - j]) for j in range(1, h + 1)]
    out = [None] * n
    acc = x[0]
    for j in range(h):
        acc = g.cadd(acc, s[j])
    out[0] = acc
    for k in range(1, h + 1):
        a = x[0]
        b = (ZERO, ZERO)
        for j in range(1, h + 1):
            ang = 2 * math.pi * j * k / n
            a = g.cadd(a, (g.scale(s[j - 1][0], math.cos(ang)), g.scale(s[j - 1][1], math.cos(ang))))
            b = g.cadd(b, (g.scale(d[j - 1][0], math.sin(ang)), g.scale(d[j - 1][1], math.sin(ang))))
        # X[k] = a + sign*i*b ; X[n-k] = a - sign*i*b
        ib = (g.scale(b[1], -sign), g.scale(b[0], sign))  # sign*i*b
        out[k] = g.cadd(a, ib)
        out[n - k] = g.csub(a, ib)
    return out


def r2c(g: Gen, x):
    """Real forward DFT, returns bins 0..n/2 (complex lazy tuples)."""
    n = len(x)
    if n == 1:
        return [(x[0], ZERO)]
    if n == 2:
        return [(g.add(x[0], x[1]), ZERO), (g.sub(x[0], x[1]), ZERO)]
    if n % 2:
        full = odd_dft(g, [(v, ZERO) for v in x], -1)
        return full[: n // 2 + 1]
    m = n // 2
    E = r2c(g, x[0::2])
    O = r2c(g, x[1::2])

    def get(H, k):
        if k <= m // 2:
            return H[k]
        return g.cconj(H[m - k])

    out = []
    for k in range(m + 1):
        e = get(E, k % m) if k < m else get(E, 0)
        o = get(O, k % m) if k < m else get(O, 0)
        t = g.cmulc(o, _w(-1, k, n))
        out.append(g.cadd(e, t))
    return out


def c2r(g: Gen, X):
    """Unnormalised inverse real DFT from bins 0..n/2 (Hermitian input)."""
    m = len(X) - 1
    n = 2 * m
    if n == 2:
        return [g.add(X[0][0], X[1][0]), g.sub(X[0][0], X[1][0])]
    half = m // 2

    def getX(k):
        return X[k]

    E, O = [], []
    for k in range(half + 1):
        a = getX(k)
        b = g.cconj(getX(m - k))
        E.append(g.cadd(a, b))
        O.append(g.cmulc(g.csub(a, b), _w(+1, k, n)))
    e = c2r(g, E)
    o = c2r(g, O)
    out = [None] * n
    for j in range(m):
        out[2 * j] = e[j]
        out[2 * j + 1] = o[j]
    return out


# ---------------------------------------------------------------------------
# emission
# ---------------------------------------------------------------------------

def _emit_nodes(g: Gen, roots):
    live = set()
    stack = [r.node for r in roots if not r.zero]
    while stack:
        n = stack.pop()
        if n.name in live or n.op == "in":
            continue
        live.add(n.name)
        stack.extend(n.args)
    lines = []
    counts = {"add": 0, "fma": 0, "mul": 0}
    for n in g.nodes:
        if n.name not in live:
            continue
        if n.op == "add":
            lines.append(f"const float {n.name} = {n.args[0].name} + {n.args[1].name};")
            counts["add"] += 1
        elif n.op == "sub":
            lines.append(f"const float {n.name} = {n.args[0].name} - {n.args[1].name};")
            counts["add"] += 1
        elif n.op == "fma":
            lines.append(f"const float {n.name} = fmaf({_f32(n.const)}, {n.args[0].name}, {n.args[1].name});")
            counts["fma"] += 1
        else:
            raise AssertionError(n.op)
    return lines, counts


def _finish(g, outs, targets):
    """Materialise outputs; returns (lines, counts)."""
    lines, counts = _emit_nodes(g, outs)
    for tgt, v in zip(targets, outs):
        e = g.expr(v)
        if not v.zero and not (_close(v.coef, 1.0) or _close(v.coef, -1.0)):
            counts["mul"] += 1
        lines.append(f"{tgt} = {e};")
    return lines, counts


def gen_r2c(n):
    g = Gen()
    x = [g.inp(f"x[{j}]") for j in range(n)]
    X = r2c(g, x)
    outs = [X[0][0], X[n // 2][0]]
    for k in range(1, n // 2):
        outs += [X[k][0], X[k][1]]
    tg = [f"y[{i}]" for i in range(n)]
    lines, counts = _finish(g, outs, tg)
    sig = f"static __device__ __forceinline__ void r2c_{n}(const float (&x)[{n}], float (&y)[{n}])"
    return sig, lines, counts


def gen_c2r(n):
    g = Gen()
    X = [(g.inp("y[0]"), ZERO)]
    for k in range(1, n // 2):
        X.append((g.inp(f"y[{2 * k}]"), g.inp(f"y[{2 * k + 1}]")))
    X.append((g.inp("y[1]"), ZERO))
    out = c2r(g, X)
    lines, counts = _finish(g, out, [f"x[{j}]" for j in range(n)])
    sig = f"static __device__ __forceinline__ void c2r_{n}(const float (&y)[{n}], float (&x)[{n}])"
    return sig, lines, counts


def gen_cdft(n, sign):
    g = Gen()
    x = [(g.inp(f"re[{j}]"), g.inp(f"im[{j}]")) for j in range(n)]
    X = cdft(g, x, sign)
    outs, tg = [], []
    for k in range(n):
        outs += [X[k][0], X[k][1]]
        tg += [f"o_re[{k}]", f"o_im[{k}]"]
    lines, counts = _finish(g, outs, tg)
    # write to temporaries first, then copy back (in place)
    lines = [f"float o_re[{n}], o_im[{n}];"] + lines
    lines += [f"#pragma unroll", f"for (int k = 0; k < {n}; ++k) {{ re[k] = o_re[k]; im[k] = o_im[k]; }}"]
    name = "fwd" if sign < 0 else "inv"
    sig = f"static __device__ __forceinline__ void cdft_{n}_{name}(float (&re)[{n}], float (&im)[{n}])"
    return sig, lines, counts


def gen_rdft_odd(n):
    g = Gen()
    x = [g.inp(f"x[{j}]") for j in range(n)]
    X = r2c(g, x)
    h = n // 2
    outs, tg = [], []
    for k in range(h + 1):
        outs.append(X[k][0])
        tg.append(f"re[{k}]")
        if k:
            outs.append(X[k][1])
            tg.append(f"im[{k}]")
    lines, counts = _finish(g, outs, tg)
    lines.append("im[0] = 0.0f;")
    sig = (f"static __device__ __forceinline__ void rdftT_{n}(const float (&x)[{n}], "
           f"float (&re)[{h + 1}], float (&im)[{h + 1}])")
    return sig, lines, counts


def all_codelets():
    out = []
    for n in (8, 16, 32):
        out.append(("r2c", n, gen_r2c(n)))
        out.append(("c2r", n, gen_c2r(n)))
        out.append(("cdft_fwd", n, gen_cdft(n, -1)))
        out.append(("cdft_inv", n, gen_cdft(n, +1)))
    out.append(("cdft_fwd", 4, gen_cdft(4, -1)))
    out.append(("cdft_inv", 4, gen_cdft(4, +1)))
    for n in (3, 5, 7):
        out.append(("cdft_fwd", n, gen_cdft(n, -1)))
        out.append(("rdftT", n, gen_rdft_odd(n)))
    return out


HEADER = """// GENERATED by gen_codelets.py -- do not edit by hand.
//
// Straight-line DFT codelets on register arrays, derived from the DFT
// definition with a lazy-coefficient radix-2 / odd-pair generator.
// Conventions: forward sign -1, inverse sign +1, no normalisation.
//   r2c_N : real -> packed [X0.re, X(N/2).re, X1.re, X1.im, ...]
//   c2r_N : packed -> real (imag of bins 0 and N/2 ignored)
//   cdft_N_fwd / cdft_N_inv : complex, in place
//   rdftT_N : real odd-length forward DFT, bins 0..N/2
#pragma once
"""


def twiddle_tables():
    """Per-T tables of w^(p*r), w = exp(+2*pi*i/T), r = (T-1)/2: the weight of
    temporal bin p in the inverse transform evaluated at the centre frame."""
    lines = ["template <int T> struct CentreTwiddle;"]
    for T in (1, 3, 5, 7):
        r = (T - 1) // 2
        re = [math.cos(2 * math.pi * p * r / T) for p in range(T)]
        im = [math.sin(2 * math.pi * p * r / T) for p in range(T)]
        re_s = ", ".join(_f32(v) for v in re)
        im_s = ", ".join(_f32(v if abs(v) > 1e-15 else 0.0) for v in im)
        lines.append(f"template <> struct CentreTwiddle<{T}> {{")
        lines.append(f"    static __device__ __forceinline__ float re(int p) {{ constexpr float v[{T}] = {{{re_s}}}; return v[p]; }}")
        lines.append(f"    static __device__ __forceinline__ float im(int p) {{ constexpr float v[{T}] = {{{im_s}}}; return v[p]; }}")
        lines.append("};")
    return lines


def half_twiddle_tables():
    """W_B^(-y) = exp(-2 pi i y / B), y < B/2: the pre-twiddle of the odd
    half of a radix-2 decimation-in-frequency split (its conjugate is the
    inverse post-twiddle)."""
    lines = ["template <int B> struct HalfTwiddle;"]
    for B in (8, 16, 32):
        M = B // 2
        re = [math.cos(2 * math.pi * y / B) for y in range(M)]
        im = [-math.sin(2 * math.pi * y / B) for y in range(M)]
        fix = lambda v: 0.0 if abs(v) < 1e-15 else v
        re_s = ", ".join(_f32(fix(v)) for v in re)
        im_s = ", ".join(_f32(fix(v)) for v in im)
        lines.append(f"template <> struct HalfTwiddle<{B}> {{")
        lines.append(f"    static __device__ __forceinline__ float re(int y) {{ constexpr float v[{M}] = {{{re_s}}}; return v[y]; }}")
        lines.append(f"    static __device__ __forceinline__ float im(int y) {{ constexpr float v[{M}] = {{{im_s}}}; return v[y]; }}")
        lines.append("};")
    return lines


def write(path):
    parts = [HEADER]
    parts += twiddle_tables()
    parts += half_twiddle_tables()
    parts.append("")
    for kind, n, (sig, lines, counts) in all_codelets():
        parts.append(f"// {kind} n={n}: {counts['add']} add, {counts['fma']} fma, {counts['mul']} mul")
        parts.append(sig + " {")
        parts += ["    " + ln for ln in lines]
        parts.append("}\n")
    with open(path, "w") as f:
        f.write("\n".join(parts))


# ---------------------------------------------------------------------------
# self check: execute emitted code in float64
# ---------------------------------------------------------------------------

def _run(lines, env):
    code = []
    for ln in lines:
        ln = ln.strip()
        if ln.startswith("float ") or ln.startswith("#pragma") or ln.startswith("for "):
            continue
        ln = ln.replace("const float ", "").rstrip(";")
        ln = ln.replace("fmaf(", "_fma(")
        ln = re.sub(r"(\d)f\b", r"\1", ln)
        code.append(ln)
    env["_fma"] = lambda a, b, c: a * b + c
    exec("\n".join(code), env)


def check():
    global _FULL_PRECISION
    _FULL_PRECISION = True
    rng = np.random.default_rng(1)
    ok = True
    for kind, n, (sig, lines, counts) in all_codelets():
        if kind == "r2c":
            x = rng.standard_normal(n)
            env = {"x": list(x), "y": [0.0] * n}
            _run(lines, env)
            X = np.fft.rfft(x)
            ref = [X[0].real, X[n // 2].real]
            for k in range(1, n // 2):
                ref += [X[k].real, X[k].imag]
            err = np.max(np.abs(np.array(env["y"]) - ref))
        elif kind == "c2r":
            y = rng.standard_normal(n)
            env = {"y": list(y), "x": [0.0] * n}
            _run(lines, env)
            X = np.zeros(n // 2 + 1, complex)
            X[0] = y[0]
            X[n // 2] = y[1]
            for k in range(1, n // 2):
                X[k] = y[2 * k] + 1j * y[2 * k + 1]
            ref = np.fft.irfft(X, n) * n
            err = np.max(np.abs(np.array(env["x"]) - ref))
        elif kind in ("cdft_fwd", "cdft_inv"):
            re = rng.standard_normal(n)
            im = rng.standard_normal(n)
            env = {"re": list(re), "im": list(im), "o_re": [0.0] * n, "o_im": [0.0] * n}
            _run(lines, env)
            z = re + 1j * im
            ref = np.fft.fft(z) if kind == "cdft_fwd" else np.fft.ifft(z) * n
            got = np.array(env["o_re"]) + 1j * np.array(env["o_im"])
            err = np.max(np.abs(got - ref))
        else:
            x = rng.standard_normal(n)
            h = n // 2
            env = {"x": list(x), "re": [0.0] * (h + 1), "im": [0.0] * (h + 1)}
            _run(lines, env)
            X = np.fft.rfft(x)
            got = np.array(env["re"]) + 1j * np.array(env["im"])
            err = np.max(np.abs(got - X[: h + 1]))
        instr = counts["add"] + counts["fma"] + counts["mul"]
        flag = "ok" if err < 1e-9 else "FAIL"
        ok &= err < 1e-9
        print(f"{kind:9s} n={n:2d}: add={counts['add']:4d} fma={counts['fma']:4d} mul={counts['mul']:3d} "
              f"instr={instr:4d} flops={counts['add'] + 2 * counts['fma'] + counts['mul']:4d} err={err:.2e} {flag}")
    return ok


if __name__ == "__main__":
    if "--check" in sys.argv:
        sys.exit(0 if check() else 1)
    here = os.path.dirname(os.path.abspath(__file__))
    write(os.path.join(here, "codelets.cuh"))
    print("wrote codelets.cuh")
