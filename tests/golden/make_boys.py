"""Generate the Boys-function fixture boys_mpmath.npz with mpmath (independent of the
reference and of the engine).

F_m(T) = int_0^1 t^(2m) exp(-T t^2) dt = 1F1(m + 1/2; m + 3/2; -T) / (2m + 1), evaluated at
40 significant digits for m = 0..10 (the orders the engine's table serves) on a grid of T
that covers:
  * T = 0 and a log-spaced range 1e-14 .. 1e3;
  * 400 seeded uniform points in [0, 36) (the tabulated Taylor region) and the grid points
    k/10 and midpoints (k + 1/2)/10 there, where the Taylor step is longest;
  * both sides of the switch to the asymptotic form at T = 36.
Values are stored as float64 (their rounding, 1.1e-16 relative, is far below the tolerances
tested).  T is stored as float64; an FP32 comparison takes T rounded to float32 and uses
the float32 entries, evaluated at that rounded T.

Usage: python tests/golden/make_boys.py
"""
import os

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MMAX = 10


def boys(m, T):
    if T == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.hyp1f1(m + mp.mpf(1) / 2, m + mp.mpf(3) / 2, -T) / (2 * m + 1)


def main():
    mp.mp.dps = 40
    rng = np.random.default_rng(20261203)
    T = [0.0]
    T += list(np.logspace(-14, 3, 69))
    T += list(rng.uniform(0.0, 36.0, size=400))
    T += [k / 10 for k in range(0, 360, 7)] + [(k + 0.5) / 10 for k in range(0, 360, 7)]
    T += [35.9, 35.95, 35.999999, 36.0, 36.000001, 36.05, 37.5, 50.0, 117.3, 999.0]
    T = np.array(sorted(set(T)), dtype=np.float64)
    T32 = T.astype(np.float32).astype(np.float64)
    F = np.array([[float(boys(m, mp.mpf(float(t)))) for m in range(MMAX + 1)] for t in T])
    F32 = np.array([[float(boys(m, mp.mpf(float(t)))) for m in range(MMAX + 1)] for t in T32])
    np.savez_compressed(os.path.join(HERE, "boys_mpmath.npz"), T=T, F=F, T32=T32, F32=F32)
    print(len(T), "points")


if __name__ == "__main__":
    main()
