"""FP64 numpy restatement of the reference's Gaussian instrumental broadening (test
infrastructure): convolve_spectra_with_gauss (cmlib/mathtools.cc:1350-1414) with its monotone
quadratic Bezier interpolation interpol_1d (cmlib/mathtools.cc:1057-1117).

Steps, as the reference takes them: a uniform fine grid from lambda_1 - 10 w to lambda_N + 10 w
with step w / 2 (rounded to a whole number of steps); the spectra interpolated onto it (constant
outside the original range); the integral with the kernel exp(-(dl/w)^2) / (sqrt(pi) w) and
trapezoid-like weights (half steps at both ends); interpolation back to the original grid.

One deliberate deviation: for the first interval of a grid interpol_1d reads its h2 before it is
set (mathtools.cc:1073, 1093: the i = 0 branch never assigns it); this restatement uses that
interval's width.  The reference's output there is undefined (values up to 1e44 were seen); the
kernel tails spread it over ~12 widths from the blue end, beyond which the two agree.
"""
import numpy as np


def interpol_bezier(f, x, xq):
    """interpol_1d for a vector of channels: f [N, C], x [N] increasing, one query point."""
    N = x.shape[0]
    if not (xq < x[N - 1] and xq > x[0]):
        return f[N - 1].copy() if xq >= x[N - 1] else f[0].copy()
    i = int(np.searchsorted(x[1:], xq, side="right"))  # first i with xq < x[i + 1]
    i = min(i, N - 2)
    if i > 0:
        h1 = x[i] - x[i - 1]
        h2 = x[i + 1] - x[i]
        d1 = (f[i] - f[i - 1]) / h1
        d2 = (f[i + 1] - f[i]) / h2
        al = (1.0 + h2 / (h1 + h2)) / 3.0
        with np.errstate(divide="ignore", invalid="ignore"):
            fd1 = np.where(d1 * d2 > 0, d1 * d2 / (al * d2 + (1.0 - al) * d1), 0.0)
    else:
        h2 = x[1] - x[0]  # see the module docstring
        fd1 = (f[1] - f[0]) / (x[1] - x[0])
        h1 = None
    C0 = f[i] + h2 * 0.5 * fd1
    if i + 1 < N - 1:
        h1 = x[i + 1] - x[i]
        h2b = x[i + 2] - x[i + 1]
        d1 = (f[i + 1] - f[i]) / h1
        d2 = (f[i + 2] - f[i + 1]) / h2b
        al = (1.0 + h2b / (h1 + h2b)) / 3.0
        with np.errstate(divide="ignore", invalid="ignore"):
            fd2 = np.where(d1 * d2 > 0, d1 * d2 / (al * d2 + (1.0 - al) * d1), 0.0)
    else:
        fd2 = (f[N - 1] - f[N - 2]) / (x[N - 1] - x[N - 2])
        if h1 is None:  # i == 0 and N == 2: h1 was never set either
            h1 = x[1] - x[0]
    C1 = f[i + 1] - h1 * 0.5 * fd2
    C = 0.5 * (C0 + C1)
    u = (xq - x[i]) / (x[i + 1] - x[i])
    return (1.0 - u) * (1.0 - u) * f[i] + u * u * f[i + 1] + u * 2.0 * (1.0 - u) * C


def fine_grid(lam, width):
    l_min = lam[0] - 10.0 * width
    l_max = lam[-1] + 10.0 * width
    n = int((l_max - l_min) / (0.5 * width)) + 1
    step = (l_max - l_min) / (n - 1)
    return l_min + np.arange(n) * step, step


def convolve_gauss(S, lam, width):
    """S [n, 4] (or [n, C]) on the grid lam [n]; returns the broadened spectra."""
    S = np.asarray(S, dtype=np.float64)
    lam = np.asarray(lam, dtype=np.float64)
    lf, step = fine_grid(lam, width)
    nf = lf.shape[0]
    Sf = np.array([interpol_bezier(S, lam, x) for x in lf])
    w = np.full(nf, step)
    w[0] = w[-1] = 0.5 * step
    K = 0.56418958354 / width * np.exp(-((lf[None, :] - lf[:, None]) ** 2) / width / width)
    Sc = (K * w[None, :]) @ Sf
    return np.array([interpol_bezier(Sc, lf, x) for x in lam])
