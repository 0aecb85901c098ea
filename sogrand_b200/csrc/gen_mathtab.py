"""Generate sg_mathtab.h: constants and tables of the decoder's own exp/log.

The decoder computes exp and log with its own table-driven routines
(Tang's method: P. T. P. Tang, "Table-driven implementation of the
exponential function in IEEE floating-point arithmetic", ACM TOMS 15(2),
1989, and the matching logarithm construction), so that host and device
evaluate them bit-identically.  Every table entry here is derived from
the mathematics with mpmath at 256-bit precision and rounded to nearest:

  exp:  H_j = RN(2^(j/128)),  t_j = RN((2^(j/128) - H_j) / H_j),  j < 128
  log:  the bit pattern of x minus that of 0.6875 is split into a binary
        exponent e and a 7-bit index j; z = x / 2^e lies in [0.6875, 1.375)
        and subinterval j has centre m_j.  c_j = RN(1/m_j) (exactly 1 on the
        two subintervals that touch 1.0, so log(x) near 1 has no cancellation),
        and -log(c_j) is stored as a double-double (hi, lo).

The correctly rounded routines of sg_crmath.h reuse both tables; their
extra constants (range limits, a three-part ln2/128, Taylor coefficients in
double-double) are derived the same way.

Run:  python gen_mathtab.py > sg_mathtab.h
"""
import struct
import mpmath as mp

mp.mp.prec = 256


def rn(v):
    """Round an mpf to the nearest binary64."""
    return float(mp.mpf(v))


def hexd(v):
    return float(v).hex()


def dd(v):
    hi = rn(v)
    lo = rn(mp.mpf(v) - mp.mpf(hi))
    return hi, lo


def bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def from_bits(b):
    return struct.unpack("<d", struct.pack("<Q", b))[0]


def main():
    out = []
    w = out.append
    w("/* Generated by gen_mathtab.py -- do not edit.  Constants and tables of")
    w(" * the decoder's own exp/log (see sg_math.h).  All values are round-to-")
    w(" * nearest binary64 images of exact quantities computed with mpmath. */")
    w("#pragma once")
    N = 128
    ln2 = mp.log(2)
    # exp range reduction: k = round(x * N / ln2), r = x - k * ln2 / N.
    inv = rn(N / ln2)
    c = ln2 / N
    # hi part keeps 35 significant bits, so k * hi is exact for |k| < 2^18.
    e = int(mp.floor(mp.log(c, 2)))
    q = mp.mpf(2) ** (e - 34)
    hi = float(mp.floor(c / q) * q)
    lo = rn(c - mp.mpf(hi))
    w("#define SG_EXP_INV_LN2_N %s  /* N/ln2, N = 128 */" % hexd(inv))
    w("#define SG_EXP_LN2_N_HI %s  /* ln2/N, 35 significant bits */" % hexd(hi))
    w("#define SG_EXP_LN2_N_LO %s  /* ln2/N - SG_EXP_LN2_N_HI */" % hexd(lo))
    w("#define SG_EXP_SHIFT 0x1.8p52")
    # Taylor coefficients 1/n! for e^r - 1 - r, n = 2..7.
    for n in range(2, 8):
        w("#define SG_EXP_C%d %s  /* 1/%d! */" % (n, hexd(rn(mp.mpf(1) / mp.factorial(n))), n))
    w("/* {H_j, t_j}: 2^(j/128) ~= H_j * (1 + t_j) */")
    w("#define SG_EXP_TAB_INIT { \\")
    rows = []
    for j in range(N):
        v = mp.mpf(2) ** (mp.mpf(j) / N)
        H = rn(v)
        t = rn((v - mp.mpf(H)) / mp.mpf(H))
        rows.append("  %s, %s" % (hexd(H), hexd(t)))
    w(", \\\n".join(rows) + " \\\n}")

    # log: OFF = bits(0.6875)
    OFF = bits(0.6875)
    w("#define SG_LOG_OFF 0x%016xULL  /* bit pattern of 0.6875 */" % OFF)
    ln2hi_e = 0
    # ln2 split: hi has 42 significant bits so e*hi is exact for |e| < 2^11.
    q = mp.mpf(2) ** (-42)
    l2hi = float(mp.floor(ln2 / q) * q)
    l2lo = rn(ln2 - mp.mpf(l2hi))
    w("#define SG_LOG_LN2_HI %s" % hexd(l2hi))
    w("#define SG_LOG_LN2_LO %s" % hexd(l2lo))
    # log1p(r) = r + r^2 * (C2 + r*C3 + ... + r^7*C9), Ck = (-1)^(k+1)/k.
    for k in range(2, 10):
        v = mp.mpf((-1) ** (k + 1)) / k
        w("#define SG_LOG_C%d %s  /* %s1/%d */" % (k, hexd(rn(v)), "-" if k % 2 == 0 else "+", k))
    w("/* {c_j, hi(-log c_j), lo(-log c_j)} for the 128 subintervals of [0.6875, 1.375) */")
    w("#define SG_LOG_TAB_INIT { \\")
    rows = []
    for j in range(N):
        lo_b = OFF + (j << 45)
        hi_b = OFF + ((j + 1) << 45)
        zlo = mp.mpf(from_bits(lo_b))
        # upper end: the interval containing 2^0 in bit space is contiguous in value
        zhi = mp.mpf(from_bits(hi_b)) if j < N - 1 else mp.mpf(1.375)
        if zlo <= 1 <= zhi or (zhi == 1) or (zlo == 1):
            cj = 1.0
        else:
            cj = rn(2 / (zlo + zhi))
        if cj == 1.0:
            h, l = 0.0, 0.0
        else:
            h, l = dd(-mp.log(mp.mpf(cj)))
        rows.append("  %s, %s, %s" % (hexd(cj), hexd(h), hexd(l)))
    w(", \\\n".join(rows) + " \\\n}")

    # ---- correctly rounded exp/log (sg_crmath.h), same tables as above
    w("/* correctly rounded exp/log (sg_crmath.h) */")
    w("#define SG_CR_EXP_XMAX %s  /* largest x with RN(exp(x)) finite */" % hexd(EXP_XMAX))
    w("#define SG_CR_EXP_XMIN %s  /* smallest x with RN(exp(x)) > 0 */" % hexd(EXP_XMIN))
    # ln2/N = C1 + C2 + C3: C1 and C2 keep 35 significant bits (k*C1, k*C2
    # exact for |k| < 2^18), C3 the rounded rest
    c = ln2 / N
    e1 = int(mp.floor(mp.log(c, 2)))
    q1 = mp.mpf(2) ** (e1 - 34)
    C1 = mp.floor(c / q1) * q1
    rest = c - C1
    e2 = int(mp.floor(mp.log(rest, 2)))
    q2 = mp.mpf(2) ** (e2 - 34)
    C2 = mp.floor(rest / q2) * q2
    C3 = rn(rest - C2)
    w("#define SG_CR_EXP_C1 %s" % hexd(float(C1)))
    w("#define SG_CR_EXP_C2 %s" % hexd(float(C2)))
    w("#define SG_CR_EXP_C3 %s" % hexd(C3))
    # 1/n!: double-double for n = 2..5, double for n = 6..11
    for n in range(2, 12):
        v = mp.mpf(1) / mp.factorial(n)
        if n <= 5:
            h, l = dd(v)
            w("#define SG_CR_EXP_F%d_HI %s" % (n, hexd(h)))
            w("#define SG_CR_EXP_F%d_LO %s" % (n, hexd(l)))
        else:
            w("#define SG_CR_EXP_F%d %s" % (n, hexd(rn(v))))
    # ln2 = SG_LOG_LN2_HI + SG_LOG_LN2_LO + SG_CR_LOG_LN2_LO2
    w("#define SG_CR_LOG_LN2_LO2 %s" % hexd(rn(ln2 - mp.mpf(l2hi) - mp.mpf(l2lo))))
    # (-1)^(n+1)/n: double for n = 2..17, double-double too for n = 2..9
    for n in range(2, 18):
        v = mp.mpf((-1) ** (n + 1)) / n
        if n <= 9:
            h, l = dd(v)
            w("#define SG_CR_LOG_G%d_HI %s" % (n, hexd(h)))
            w("#define SG_CR_LOG_G%d_LO %s" % (n, hexd(l)))
        w("#define SG_CR_LOG_G%d %s" % (n, hexd(rn(v))))
    print("\n".join(out))


def _exp_limits():
    """Largest x with RN(exp(x)) finite and smallest x with RN(exp(x)) > 0."""
    dmax = from_bits(0x7FEFFFFFFFFFFFFF)
    top = mp.mpf(dmax) + mp.mpf(2) ** (1023 - 53)
    x = float(mp.log(top))
    while mp.exp(mp.mpf(x)) >= top:
        x = from_bits(bits(x) - 1)
    while mp.exp(mp.mpf(from_bits(bits(x) + 1))) < top:
        x = from_bits(bits(x) + 1)
    xmax = x
    bot = mp.mpf(2) ** -1075
    x = float(mp.log(bot))
    while mp.exp(mp.mpf(x)) <= bot:
        x = from_bits(bits(x) - 1)
    while mp.exp(mp.mpf(from_bits(bits(x) + 1))) > bot:
        x = from_bits(bits(x) + 1)
    return xmax, x


EXP_XMAX, EXP_XMIN = _exp_limits()


if __name__ == "__main__":
    main()
