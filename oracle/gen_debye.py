"""Generate the Debye polynomials u_1..u_13 used by the uniform asymptotic
expansion of I_v(x) (DLMF 10.41.10; Abramowitz & Stegun 9.3.9/9.3.10).

Recurrence (exact, rational arithmetic):
    u_0(t) = 1
    u_{k+1}(t) = 1/2 t^2 (1 - t^2) u_k'(t) + 1/8 Int_0^t (1 - 5 s^2) u_k(s) ds

u_k(t) = t^k * P_k(t^2), P_k of degree k.  The output header stores the
coefficients of P_k (ascending powers of t^2) as doubles, one row per k.
Run:  python oracle/gen_debye.py > oracle/debye_coeffs.h
"""
from fractions import Fraction


def debye(kmax):
    u = [[Fraction(1)]]  # coefficient list in powers of t
    for k in range(kmax):
        c = u[-1]
        deg = len(c) - 1
        # derivative
        d = [c[i] * i for i in range(1, deg + 1)]  # coeff of t^(i-1)
        nxt = [Fraction(0)] * (deg + 4)
        # 1/2 t^2 (1 - t^2) u'
        for i, a in enumerate(d):      # a * t^i
            nxt[i + 2] += a / 2
            nxt[i + 4] -= a / 2
        # 1/8 int_0^t (1 - 5 s^2) u ds
        for i, a in enumerate(c):
            nxt[i + 1] += a / 8 / (i + 1)
            nxt[i + 3] += -5 * a / 8 / (i + 3)
        while nxt and nxt[-1] == 0:
            nxt.pop()
        u.append(nxt)
    return u


def main():
    kmax = 13
    u = debye(kmax)
    print("/* Generated by oracle/gen_debye.py: Debye polynomials u_k(t) = t^k P_k(t^2),")
    print("   DEBYE_P[k][j] = coefficient of t^(2j) in P_k, k = 1..13 (row 0 unused). */")
    print("#ifndef TCE_DEBYE_COEFFS_H\n#define TCE_DEBYE_COEFFS_H")
    print("#define DEBYE_KMAX %d" % kmax)
    print("static const double DEBYE_P[%d][%d] = {" % (kmax + 1, kmax + 1))
    for k in range(kmax + 1):
        c = u[k]
        row = []
        for j in range(kmax + 1):
            idx = k + 2 * j
            if k > 0 and idx < len(c):
                row.append(c[idx])
            else:
                row.append(Fraction(0))
            # all odd-offset coefficients must vanish
        for idx, a in enumerate(c):
            if k > 0 and (idx - k) % 2 != 0:
                assert a == 0
        print("  {" + ", ".join("%.17g" % float(a) for a in row) + "},")
    print("};\n#endif")


if __name__ == "__main__":
    main()
