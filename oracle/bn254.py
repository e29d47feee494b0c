"""BN254 optimal-ate pairing and the Groth16 verification equation, pure Python.

TEST INFRASTRUCTURE ONLY (the reference verifies proofs by calling snarkjs, which is not
vendored; this is the independent check that every proof the GPU prover makes verifies).

Published algorithm, restated: Fq12 is represented as Fq[w]/(w^12 - 18 w^6 + 82) (w^6 =
9 + u with u^2 = -1), G2 points on the sextic twist y^2 = x^3 + 3/(9+u) are mapped into
E(Fq12) by x -> x w^2, y -> y w^3; the Miller loop runs over the bits of 6x + 2
(x = 4965661367192848881) with affine line functions, adds the Frobenius images
pi(Q) and -pi^2(Q), and the final exponentiation raises to (q^12 - 1)/r.
"""
from __future__ import annotations

Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
ATE_LOOP = 29793968203157093288
LOG_ATE = 63
MOD12 = [82, 0, 0, 0, 0, 0, Q - 18, 0, 0, 0, 0, 0]  # w^12 = 18 w^6 - 82


def _inv(a: int) -> int:
    return pow(a, Q - 2, Q)


class F12:
    __slots__ = ("c",)

    def __init__(self, c):
        self.c = [x % Q for x in c]

    @staticmethod
    def one():
        return F12([1] + [0] * 11)

    @staticmethod
    def const(a):
        return F12([a] + [0] * 11)

    def __add__(self, o):
        return F12([a + b for a, b in zip(self.c, o.c)])

    def __sub__(self, o):
        return F12([a - b for a, b in zip(self.c, o.c)])

    def __neg__(self):
        return F12([-a for a in self.c])

    def scale(self, k):
        return F12([a * k for a in self.c])

    def __mul__(self, o):
        if isinstance(o, int):
            return self.scale(o)
        b = [0] * 23
        for i, x in enumerate(self.c):
            if x:
                for j, y in enumerate(o.c):
                    b[i + j] += x * y
        # reduce with w^12 = 18 w^6 - 82
        for k in range(22, 11, -1):
            t = b[k]
            if t:
                b[k] = 0
                b[k - 6] += 18 * t
                b[k - 12] -= 82 * t
        return F12(b[:12])

    def __eq__(self, o):
        return self.c == o.c

    def __pow__(self, e):
        res, base = F12.one(), self
        while e:
            if e & 1:
                res = res * base
            base = base * base
            e >>= 1
        return res

    def inv(self):
        """Extended Euclid in Fq[w] modulo w^12 - 18 w^6 + 82."""
        r0 = [82, 0, 0, 0, 0, 0, Q - 18, 0, 0, 0, 0, 0, 1]
        r1 = _trim(list(self.c))
        s0, s1 = [0], [1]
        while len(r1) > 1:
            q, rem = _divmod(r0, r1)
            r0, r1 = r1, rem
            s0, s1 = s1, _psub(s0, _pmul(q, s1))
        c = _inv(r1[0])
        s1 = s1 + [0] * (12 - len(s1))
        return F12([x * c for x in s1[:12]])

    def __truediv__(self, o):
        return self * o.inv()


def _trim(p):
    p = [x % Q for x in p]
    while len(p) > 1 and p[-1] == 0:
        p.pop()
    return p


def _psub(a, b):
    n = max(len(a), len(b))
    return _trim([(a[i] if i < len(a) else 0) - (b[i] if i < len(b) else 0) for i in range(n)])


def _pmul(a, b):
    out = [0] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        if x:
            for j, y in enumerate(b):
                out[i + j] += x * y
    return _trim(out)


def _divmod(a, b):
    a = _trim(list(a))
    b = _trim(list(b))
    inv_lead = _inv(b[-1])
    q = [0] * max(1, len(a) - len(b) + 1)
    rem = list(a)
    for i in range(len(a) - len(b), -1, -1):
        coef = rem[i + len(b) - 1] * inv_lead % Q
        q[i] = coef
        if coef:
            for j, y in enumerate(b):
                rem[i + j] = (rem[i + j] - coef * y) % Q
    return _trim(q), _trim(rem[:len(b) - 1] if len(b) > 1 else [0])


def _fq2_to_f12_twisted(xc0, xc1, yc0, yc1):
    """G2 point (x, y) over Fq2 -> E(Fq12) through the twist."""
    # Fq2 element a + b u maps to (a - 9 b) + b w^6
    nx = F12([(xc0 - 9 * xc1)] + [0] * 5 + [xc1] + [0] * 5)
    ny = F12([(yc0 - 9 * yc1)] + [0] * 5 + [yc1] + [0] * 5)
    w2 = F12([0, 0, 1] + [0] * 9)
    w3 = F12([0, 0, 0, 1] + [0] * 8)
    return (nx * w2, ny * w3)


def _line(p1, p2, t):
    x1, y1 = p1
    x2, y2 = p2
    xt, yt = t
    if x1 != x2:
        m = (y2 - y1) / (x2 - x1)
        return m * (xt - x1) - (yt - y1)
    if y1 == y2:
        m = (x1 * x1).scale(3) / (y1.scale(2))
        return m * (xt - x1) - (yt - y1)
    return xt - x1


def _add(p1, p2):
    if p1 is None:
        return p2
    if p2 is None:
        return p1
    x1, y1 = p1
    x2, y2 = p2
    if x1 == x2:
        if y1 == y2:
            m = (x1 * x1).scale(3) / (y1.scale(2))
        else:
            return None
    else:
        m = (y2 - y1) / (x2 - x1)
    x3 = m * m - x1 - x2
    return (x3, m * (x1 - x3) - y1)


def _frob(p):
    x, y = p
    return (x ** Q, y ** Q)


def miller(g2, g1):
    """Miller loop value f_{6x+2,Q}(P) with the two Frobenius correction lines (no final exp).
    g1 = (x, y) ints (normal form) or None; g2 = ((x0, x1), (y0, y1)) ints or None."""
    if g1 is None or g2 is None:
        return F12.one()
    Qp = _fq2_to_f12_twisted(g2[0][0], g2[0][1], g2[1][0], g2[1][1])
    P = (F12.const(g1[0]), F12.const(g1[1]))
    Rp, f = Qp, F12.one()
    for i in range(LOG_ATE, -1, -1):
        f = f * f * _line(Rp, Rp, P)
        Rp = _add(Rp, Rp)
        if ATE_LOOP & (1 << i):
            f = f * _line(Rp, Qp, P)
            Rp = _add(Rp, Qp)
    Q1 = _frob(Qp)
    nQ2 = _frob(Q1)
    nQ2 = (nQ2[0], -nQ2[1])
    f = f * _line(Rp, Q1, P)
    Rp = _add(Rp, Q1)
    f = f * _line(Rp, nQ2, P)
    return f


def final_exp(f: F12) -> F12:
    return f ** ((Q ** 12 - 1) // R)


def pairing(g2, g1) -> F12:
    return final_exp(miller(g2, g1))


# ------------------------------------------------------------------ group helpers ----
def g1_add(p, q):
    if p is None:
        return q
    if q is None:
        return p
    (x1, y1), (x2, y2) = p, q
    if x1 == x2:
        if (y1 + y2) % Q == 0:
            return None
        m = 3 * x1 * x1 * _inv(2 * y1) % Q
    else:
        m = (y2 - y1) * _inv((x2 - x1) % Q) % Q
    x3 = (m * m - x1 - x2) % Q
    return (x3, (m * (x1 - x3) - y1) % Q)


def g1_mul(p, k):
    acc = None
    k %= R
    while k:
        if k & 1:
            acc = g1_add(acc, p)
        p = g1_add(p, p)
        k >>= 1
    return acc


def g1_neg(p):
    return None if p is None else (p[0], (-p[1]) % Q)


def on_curve_g1(p):
    return p is None or (p[1] * p[1] - p[0] ** 3 - 3) % Q == 0


def groth16_verify(vk: dict, proof: dict, public: list) -> bool:
    """e(A, B) == e(alpha, beta) e(sum_i pub_i IC_i, gamma) e(C, delta); all points as
    normal-form ints (G1 (x, y), G2 ((x0, x1), (y0, y1)), None = infinity); public[0] = 1."""
    acc = None
    for k, ic in zip(public, vk["IC"]):
        acc = g1_add(acc, g1_mul(ic, k))
    f = miller(proof["B"], proof["A"])
    f = f * miller(vk["beta_2"], g1_neg(vk["alpha_1"]))
    f = f * miller(vk["gamma_2"], g1_neg(acc))
    f = f * miller(vk["delta_2"], g1_neg(proof["C"]))
    return final_exp(f) == F12.one()
