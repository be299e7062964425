"""Operation count of one dynamic Stokes evaluation (test infrastructure).

The assembly's algorithmic work is E = NBE*(NBE-1)*NPG^2 evaluations of the
Stokes fundamental solution per frequency, each followed by its Gauss-weighted
accumulation into the element's 3x3 H and G blocks.  This module restates
that per-Gauss-point body of the oracle (bem_oracle.c: solfund + stokes, after
src/Solfund.for:18-60, and the accumulation of src/Nonsingd.for:112-117) on a
scalar type that counts its operations, so that the flops per evaluation
(FLOP_S) are frozen from the arithmetic the reference specifies rather than
from any one implementation of it.

Counting convention (real operations):
  +, -, *, /, sqrt           1 each
  complex + complex          2       complex * complex   6 (4 mul, 2 add)
  real * complex             2       complex / real      2
  complex / complex          11 (|d|^2: 3; two numerators: 6; two divisions)
  real / complex             7 (|d|^2: 3; two products: 2; two divisions)
  cexp(z)                    1 exp call + 1 sincos call + 2 mul
Transcendental calls are tallied apart from the flops.  Products with the
Kronecker delta are structural (the delta term is added on the diagonal only),
the loop-invariant 1/(4 pi) and the subexpressions the oracle writes more than
once (cappa/r, r*r) are formed once, and products of reals are formed before
they meet a complex factor; everything else follows the oracle's expressions
operation for operation.

The Gauss-point geometry (bilinear shape functions, Jacobian, det;
bem_oracle.c gauss_point after src/Nonsingd.for:58-105) depends on the
element and the Gauss point only, not on the collocation point, so it is
counted separately (FLOP_G per element and Gauss point).
"""
from __future__ import annotations

import cmath
import math

KINDS = ("add", "mul", "div", "sqrt", "exp", "sincos")


class Tally:
    def __init__(self):
        self.n = dict.fromkeys(KINDS, 0)

    def flops(self) -> int:
        return self.n["add"] + self.n["mul"] + self.n["div"] + self.n["sqrt"]


T = Tally()


class R:
    """A counted real."""
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = float(v)

    def _o(self, o):
        return o if isinstance(o, (R, C)) else R(o)

    def __add__(self, o):
        o = self._o(o)
        if isinstance(o, C):
            return o + self
        T.n["add"] += 1
        return R(self.v + o.v)

    __radd__ = __add__

    def __sub__(self, o):
        o = self._o(o)
        if isinstance(o, C):
            return (-o) + self
        T.n["add"] += 1
        return R(self.v - o.v)

    def __rsub__(self, o):
        return self._o(o) - self

    def __neg__(self):
        return R(-self.v)  # a sign flip, folded into the consumer

    def __mul__(self, o):
        o = self._o(o)
        if isinstance(o, C):
            return o * self
        T.n["mul"] += 1
        return R(self.v * o.v)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = self._o(o)
        if isinstance(o, C):
            # real / complex
            den = o.re * o.re + o.im * o.im
            return C((self * o.re) / den, -(self * o.im) / den)
        T.n["div"] += 1
        return R(self.v / o.v)

    def __rtruediv__(self, o):
        return self._o(o) / self


class C:
    """A counted complex (a pair of counted reals)."""
    __slots__ = ("re", "im")

    def __init__(self, re, im=0.0):
        self.re = re if isinstance(re, R) else R(re)
        self.im = im if isinstance(im, R) else R(im)

    @property
    def value(self) -> complex:
        return complex(self.re.v, self.im.v)

    def __add__(self, o):
        if isinstance(o, C):
            return C(self.re + o.re, self.im + o.im)
        return C(self.re + o, self.im)

    __radd__ = __add__

    def __neg__(self):
        return C(-self.re, -self.im)

    def __sub__(self, o):
        if isinstance(o, C):
            return C(self.re - o.re, self.im - o.im)
        return C(self.re - o, self.im)

    def __rsub__(self, o):
        return (-self) + o

    def __mul__(self, o):
        if isinstance(o, C):
            return C(self.re * o.re - self.im * o.im, self.re * o.im + self.im * o.re)
        return C(self.re * o, self.im * o)

    __rmul__ = __mul__

    def __truediv__(self, o):
        if isinstance(o, C):
            den = o.re * o.re + o.im * o.im
            return C((self.re * o.re + self.im * o.im) / den,
                     (self.im * o.re - self.re * o.im) / den)
        return C(self.re / o, self.im / o)

    def __rtruediv__(self, o):
        return (o if isinstance(o, R) else R(o)) / self


def cexp(z: C) -> C:
    T.n["exp"] += 1
    T.n["sincos"] += 1
    e = R(math.exp(z.re.v))
    return C(e * R(math.cos(z.im.v)), e * R(math.sin(z.im.v)))


def _consts(zge, zcs, zcp, fr):
    """bem_oracle.c make_dyn: per frequency, not counted."""
    pi = 4.0 * math.atan(1.0)
    zwi = 1j * fr
    return {"zc0": 1.0 / ((4.0 * pi) * zge), "zc1": (zcp / zcs) ** 2, "zc2": (zcs / zcp) ** 2,
            "zkp": -zwi / zcp, "zks": -zwi / zcs, "pi": pi}


def _radial(k, r):
    """bem_oracle.c stokes (src/Solfund.for:36-49)."""
    zkp, zks, zc2 = C(k["zkp"].real, k["zkp"].imag), C(k["zks"].real, k["zks"].imag), \
        C(k["zc2"].real, k["zc2"].imag)
    zzp, zzs = zkp * r, zks * r
    zezp, zezs = cexp(zzp), cexp(zzs)
    zp2, zs2 = zzp * zzp, zzs * zzs
    fhi = (1.0 + 1.0 / zs2 - 1.0 / zzs) * zezs / r - zc2 * (1.0 / zp2 - 1.0 / zzp) * zezp / r
    cappa = (1.0 + 3.0 / zs2 - 3.0 / zzs) * zezs / r - zc2 * (1.0 + 3.0 / zp2 - 3.0 / zzp) * zezp / r
    rr = r * r
    fhidr = (-2.0 + zzs + 3.0 / zzs - 3.0 / zs2) * zezs / rr - \
        zc2 * (-1.0 + 3.0 / zzp - 3.0 / zp2) * zezp / rr
    cappadr = (zzs - 4.0 + 9.0 / zzs - 9.0 / zs2) * zezs / rr - \
        zc2 * (zzp - 4.0 + 9.0 / zzp - 9.0 / zp2) * zezp / rr
    cr = cappa / r
    aa = fhidr - cr
    bb = 4.0 * cr - 2.0 * cappadr
    zc1 = C(k["zc1"].real, k["zc1"].imag)
    cc = (zc1 - 2.0) * (aa + 0.5 * bb - 3.0 * cr) - 2.0 * cr
    return fhi, cappa, aa, bb, cc


def stokes_eval(p, g, rn, zge, zcs, zcp, fr, p12, zh=None, zg=None):
    """One evaluation: SOLFUND at Gauss point g for collocation point p with
    normal rn, then zh += zt*p12 and zg += zu*p12 (counted).  Returns the
    counted (zu, zt) as complex 3x3 lists, zu[j][i] == ZU(I,J)."""
    k = _consts(zge, zcs, zcp, fr)
    r1, r2, r3 = R(g[0]) - R(p[0]), R(g[1]) - R(p[1]), R(g[2]) - R(p[2])
    T.n["sqrt"] += 1
    rs = r1 * r1 + r2 * r2 + r3 * r3
    r = R(math.sqrt(rs.v))
    n = [R(x) for x in rn]
    drn = (r1 * n[0] + r2 * n[1] + r3 * n[2]) / r
    rd = [r1 / r, r2 / r, r3 / r]
    fhi, cappa, aa, bb, cc = _radial(k, r)
    zc0 = C(k["zc0"].real, k["zc0"].imag)
    q = R(1.0) / (R(4.0) * R(k["pi"]))
    zu = [[None] * 3 for _ in range(3)]
    zt = [[None] * 3 for _ in range(3)]
    w = R(p12)
    for j in range(3):
        for i in range(3):
            u = -(cappa * (rd[j] * rd[i]))
            if i == j:
                u = fhi + u
            zu[j][i] = zc0 * u
            a = rd[j] * n[i]
            if i == j:
                a = drn + a
            t = aa * a + bb * (rd[i] * rd[j] * drn) + cc * (rd[i] * n[j])
            zt[j][i] = t * q
            if zh is not None:
                zh[j][i] = zh[j][i] + zt[j][i] * w
                zg[j][i] = zg[j][i] + zu[j][i] * w
    return zu, zt


def gauss_geometry(co, g1, g2):
    """bem_oracle.c gauss_point (counted): (xg, yg, zg, det)."""
    g1, g2 = R(g1), R(g2)
    sp, sm = R(1.0) + g2, R(1.0) - g2
    rp, rm = R(1.0) + g1, R(1.0) - g1
    q = R(0.25)
    p = [[-(q * sm), q * sm, q * sp, -(q * sp)], [-(q * rm), -(q * rp), q * rp, q * rm]]
    f = [q * rm * sm, q * rp * sm, q * rp * sp, q * rm * sp]
    cor = [[R(x) for x in row] for row in co]
    xj = [[None] * 3 for _ in range(2)]
    for i in range(2):
        for j in range(3):
            t = p[i][0] * cor[0][j]
            for kk in range(1, 4):
                t = t + p[i][kk] * cor[kk][j]
            xj[i][j] = t
    d1 = xj[0][1] * xj[1][2] - xj[1][1] * xj[0][2]
    d2 = xj[1][0] * xj[0][2] - xj[0][0] * xj[1][2]
    d3 = xj[0][0] * xj[1][1] - xj[1][0] * xj[0][1]
    T.n["sqrt"] += 1
    s = d1 * d1 + d2 * d2 + d3 * d3
    det = R(math.sqrt(s.v))
    xyz = []
    for c in range(3):
        t = cor[0][c] * f[0]
        for kk in range(1, 4):
            t = t + cor[kk][c] * f[kk]
        xyz.append(t)
    return xyz[0], xyz[1], xyz[2], det


def count_stokes(**kw) -> dict:
    """Tally of one stokes_eval with accumulation, on representative inputs."""
    global T
    T = Tally()
    zero = [[C(0.0) for _ in range(3)] for _ in range(3)]
    zh = [row[:] for row in zero]
    zg = [row[:] for row in zero]
    args = dict(p=(0.3, -0.2, 0.0), g=(1.1, 0.7, -0.4), rn=(0.0, 0.0, 1.0),
                zge=complex(1.0, 0.02), zcs=cmath.sqrt(complex(1.0, 0.02)),
                zcp=cmath.sqrt(complex(1.0, 0.02)) * math.sqrt(3.0), fr=2.0, p12=0.37)
    args.update(kw)
    stokes_eval(**args, zh=zh, zg=zg)
    out = dict(T.n)
    out["flops"] = T.flops()
    return out


def count_geometry() -> dict:
    global T
    T = Tally()
    gauss_geometry([(0.0, 0.0, 0.0), (1.0, 0.1, 0.0), (1.1, 1.0, 0.05), (-0.1, 0.9, 0.0)], 0.3, -0.6)
    out = dict(T.n)
    out["flops"] = T.flops()
    return out


if __name__ == "__main__":
    print("per Stokes evaluation:", count_stokes())
    print("per element and Gauss point (geometry):", count_geometry())
