#!/usr/bin/env python3
"""Generates codelets.cuh: straight-line register DFT butterflies for the radix menu.

Each codelet computes the forward R-point DFT  X[k] = sum_j x[j] exp(-2 pi i jk / R)
in place on an array of R complex values held in registers. The backward
transform is obtained by the kernels through conjugation of the input and the
output, so only the forward codelets are generated.

* R = 2, 4, 8, 16: split-radix decimation-in-time network,
  X[k] = E[k] + W^k O1[k] + W^3k O3[k] with E the half-length DFT of the even
  inputs and O1, O3 the quarter-length DFTs of inputs 1 and 3 mod 4, which
  needs fewer real operations than the radix-2 network; twiddles W_R^k with
  k in {0, R/4} are applied as sign swaps, k in {R/8, 3R/8} with one
  multiply by sqrt(1/2) per component.
* R = 3, 5, 7, 11, 13: the symmetric-pair form
  X[k] = x0 + sum_j a_j cos(2 pi jk/R) - i sum_j b_j sin(2 pi jk/R),
  X[R-k] = the same with +i, where a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}.

All constants are evaluated with mpmath at 40 digits and printed with 17
significant digits (exact round-trip for IEEE double); the float kernels round
them once more at compile time.

Usage: python gen_codelets.py > codelets.cuh
"""
import mpmath

mpmath.mp.dps = 40
RADICES_POW2 = [2, 4, 8, 16]
RADICES_ODD = [3, 5, 7, 11, 13]


def lit(x):
    v = float(x)
    if v == 0.0:
        return "T(0)"
    return "T(%s)" % repr(v)


class Emitter:
    def __init__(self):
        self.lines = []
        self.count = 0

    def tmp(self, expr_re, expr_im):
        name = "t%d" % self.count
        self.count += 1
        self.lines.append("    const T %s_r = %s, %s_i = %s;" % (name, expr_re, name, expr_im))
        return name


def twiddle(em, o, m, n):
    """(re, im) expressions of W_n^m * o, W = exp(-2 pi i / n)."""
    m %= n
    if m == 0:
        return "%s_r" % o, "%s_i" % o
    if 4 * m == n:  # -i
        return "%s_i" % o, "-%s_r" % o
    if 8 * m == n:  # (1 - i)/sqrt2
        h = lit(mpmath.sqrt(2) / 2)
        t = em.tmp("%s * (%s_r + %s_i)" % (h, o, o), "%s * (%s_i - %s_r)" % (h, o, o))
        return "%s_r" % t, "%s_i" % t
    if 8 * m == 3 * n:  # -(1 + i)/sqrt2
        h = lit(mpmath.sqrt(2) / 2)
        t = em.tmp("%s * (%s_i - %s_r)" % (h, o, o), "-%s * (%s_r + %s_i)" % (h, o, o))
        return "%s_r" % t, "%s_i" % t
    ang = 2 * mpmath.pi * m / n
    c, s = lit(mpmath.cos(ang)), lit(mpmath.sin(ang))
    # (or + i oi)(c - i s) = (or c + oi s) + i (oi c - or s)
    t = em.tmp("fma(%s, %s_r, %s * %s_i)" % (c, o, s, o), "fma(%s, %s_i, -(%s * %s_r))" % (c, o, s, o))
    return "%s_r" % t, "%s_i" % t


def gen_pow2_split(R):
    em = Emitter()

    def rec(idx):
        n = len(idx)
        if n == 1:
            return [em.tmp("v[%d].x" % idx[0], "v[%d].y" % idx[0])]
        if n == 2:
            a, b = rec(idx[:1]), rec(idx[1:])
            return [em.tmp("%s_r + %s_r" % (a[0], b[0]), "%s_i + %s_i" % (a[0], b[0])),
                    em.tmp("%s_r - %s_r" % (a[0], b[0]), "%s_i - %s_i" % (a[0], b[0]))]
        e = rec(idx[0::2])
        o1 = rec(idx[1::4])
        o3 = rec(idx[3::4])
        q = n // 4
        out = [None] * n
        for k in range(q):
            ar, ai = twiddle(em, o1[k], k, n)
            br, bi = twiddle(em, o3[k], 3 * k, n)
            sm = em.tmp("%s + %s" % (ar, br), "%s + %s" % (ai, bi))
            df = em.tmp("%s - %s" % (ar, br), "%s - %s" % (ai, bi))
            out[k] = em.tmp("%s_r + %s_r" % (e[k], sm), "%s_i + %s_i" % (e[k], sm))
            out[k + 2 * q] = em.tmp("%s_r - %s_r" % (e[k], sm), "%s_i - %s_i" % (e[k], sm))
            # E[k + n/4] -/+ i d
            out[k + q] = em.tmp("%s_r + %s_i" % (e[k + q], df), "%s_i - %s_r" % (e[k + q], df))
            out[k + 3 * q] = em.tmp("%s_r - %s_i" % (e[k + q], df), "%s_i + %s_r" % (e[k + q], df))
        return out

    outs = rec(list(range(R)))
    return em.lines + ["    v[%d].x = %s_r; v[%d].y = %s_i;" % (k, o, k, o) for k, o in enumerate(outs)]


def gen_pow2(R):
    em = Emitter()
    # leaves are input registers v[j]
    def load(j):
        return em.tmp("v[%d].x" % j, "v[%d].y" % j)

    def rec(idx):
        n = len(idx)
        if n == 1:
            return [load(idx[0])]
        even = rec(idx[0::2])
        odd = rec(idx[1::2])
        out = [None] * n
        for k in range(n // 2):
            o = odd[k]
            # t = W_n^k * o, W = exp(-2 pi i k / n) = c - i s
            if k == 0:
                tr, ti = "%s_r" % o, "%s_i" % o
            elif 4 * k == n:  # -i
                tr, ti = "%s_i" % o, "-%s_r" % o
            elif 8 * k == n:  # (1 - i)/sqrt2
                h = lit(mpmath.sqrt(2) / 2)
                t = em.tmp("%s * (%s_r + %s_i)" % (h, o, o), "%s * (%s_i - %s_r)" % (h, o, o))
                tr, ti = "%s_r" % t, "%s_i" % t
            elif 8 * k == 3 * n:  # -(1 + i)/sqrt2
                h = lit(mpmath.sqrt(2) / 2)
                t = em.tmp("%s * (%s_i - %s_r)" % (h, o, o), "-%s * (%s_r + %s_i)" % (h, o, o))
                tr, ti = "%s_r" % t, "%s_i" % t
            else:
                ang = 2 * mpmath.pi * k / n
                c, s = lit(mpmath.cos(ang)), lit(mpmath.sin(ang))
                # (or + i oi)(c - i s) = (or c + oi s) + i (oi c - or s)
                t = em.tmp("fma(%s, %s_r, %s * %s_i)" % (c, o, s, o),
                           "fma(%s, %s_i, -(%s * %s_r))" % (c, o, s, o))
                tr, ti = "%s_r" % t, "%s_i" % t
            e = even[k]
            out[k] = em.tmp("%s_r + %s" % (e, tr), "%s_i + %s" % (e, ti))
            out[k + n // 2] = em.tmp("%s_r - %s" % (e, tr), "%s_i - %s" % (e, ti))
        return out

    outs = rec(list(range(R)))
    body = em.lines + ["    v[%d].x = %s_r; v[%d].y = %s_i;" % (k, o, k, o) for k, o in enumerate(outs)]
    return body


def gen_odd(R):
    h = (R - 1) // 2
    L = []
    for j in range(1, h + 1):
        L.append("    const T a%d_r = v[%d].x + v[%d].x, a%d_i = v[%d].y + v[%d].y;" % (j, j, R - j, j, j, R - j))
        L.append("    const T b%d_r = v[%d].x - v[%d].x, b%d_i = v[%d].y - v[%d].y;" % (j, j, R - j, j, j, R - j))
    L.append("    const T x0_r = v[0].x, x0_i = v[0].y;")
    sum_r = " + ".join("a%d_r" % j for j in range(1, h + 1))
    sum_i = " + ".join("a%d_i" % j for j in range(1, h + 1))
    for k in range(1, h + 1):
        ar, ai, br, bi = "x0_r", "x0_i", None, None
        for j in range(1, h + 1):
            m = (j * k) % R
            c = lit(mpmath.cos(2 * mpmath.pi * m / R))
            s = lit(mpmath.sin(2 * mpmath.pi * m / R))
            ar = "fma(%s, a%d_r, %s)" % (c, j, ar)
            ai = "fma(%s, a%d_i, %s)" % (c, j, ai)
            br = "%s * b%d_r" % (s, j) if br is None else "fma(%s, b%d_r, %s)" % (s, j, br)
            bi = "%s * b%d_i" % (s, j) if bi is None else "fma(%s, b%d_i, %s)" % (s, j, bi)
        L.append("    const T A%d_r = %s, A%d_i = %s;" % (k, ar, k, ai))
        L.append("    const T B%d_r = %s, B%d_i = %s;" % (k, br, k, bi))
    L.append("    v[0].x = x0_r + %s; v[0].y = x0_i + %s;" % (sum_r, sum_i))
    for k in range(1, h + 1):
        # X[k] = A - i B = (A_r + B_i, A_i - B_r); X[R-k] = A + i B
        L.append("    v[%d].x = A%d_r + B%d_i; v[%d].y = A%d_i - B%d_r;" % (k, k, k, k, k, k))
        L.append("    v[%d].x = A%d_r - B%d_i; v[%d].y = A%d_i + B%d_r;" % (R - k, k, k, R - k, k, k))
    return L


def main():
    out = []
    out.append("// GENERATED by gen_codelets.py -- do not edit by hand.")
    out.append("// Forward R-point DFT butterflies on registers (see the generator's docstring).")
    out.append("#pragma once")
    out.append("")
    out.append("namespace fftz {")
    out.append("template <int R> struct Dft;")
    for R in sorted(RADICES_POW2 + RADICES_ODD):
        body = gen_pow2_split(R) if R in RADICES_POW2 else gen_odd(R)
        out.append("template <> struct Dft<%d> {" % R)
        out.append("  template <typename T, typename T2>")
        out.append("  static __device__ __forceinline__ void apply(T2 (&v)[%d]) {" % R)
        out.extend("  " + l for l in body)
        out.append("  }")
        out.append("};")
    out.append("}  // namespace fftz")
    print("\n".join(out))


if __name__ == "__main__":
    main()
