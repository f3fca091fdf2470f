"""CPU restatement of tamc-pt-opt's ladder update (TEST INFRASTRUCTURE ONLY).

pt_optimize_beta, src/bin/tamc-pt-opt.rs:59-181, one iteration, in float32
with the reference's operation order:
  * StepwiseMeasure / finite_differences / monotonic_divisions (nested
    bisection) from tamc-core/src/util.rs:5-137;
  * ndarray 0.15 `sum()` of contiguous f32 data as its eight-way unrolled fold
    (numeric_util::unrolled_fold; ndarray is not vendored);
  * interp 0.1.x `interp` (not vendored): the segment that starts at the last
    knot strictly below the point among all but the last knot, else the first,
    as slope * x + intercept;
  * f32::exp / ln / log10 as glibc's expf / logf / log10f (through ctypes).
Parity of the last two items with the real crates is unpinned.  Imported only
by tests/.
"""
from __future__ import annotations

import ctypes

import numpy as np

_m = ctypes.CDLL("libm.so.6")
for _name in ("expf", "logf", "log10f", "sqrtf"):
    getattr(_m, _name).restype = ctypes.c_float
    getattr(_m, _name).argtypes = [ctypes.c_float]

F = np.float32


def expf(x):
    return F(_m.expf(float(x)))


def logf(x):
    return F(_m.logf(float(x)))


def log10f(x):
    return F(_m.log10f(float(x)))


def nd_sum(xs):
    """ndarray's unrolled_fold(xs, 0.0, +) in f32."""
    acc = F(0)
    p = [F(0)] * 8
    xs = list(xs)
    k = 0
    while len(xs) - k >= 8:
        for j in range(8):
            p[j] = F(p[j] + xs[k + j])
        k += 8
    acc = F(acc + F(p[0] + p[4]))
    acc = F(acc + F(p[1] + p[5]))
    acc = F(acc + F(p[2] + p[6]))
    acc = F(acc + F(p[3] + p[7]))
    for x in xs[k:]:
        acc = F(acc + x)
    return acc


def finite_differences(x, y):
    n = len(x)
    dx = [F(x[i + 1] - x[i]) for i in range(n - 1)]
    dy = [F(y[i + 1] - y[i]) for i in range(n - 1)]
    d = [F(0)] * n
    d[0] = F(dy[0] / dx[0])
    d[n - 1] = F(dy[-1] / dx[-1])
    for i in range(1, n - 1):
        a = F(F(dy[i - 1] * dx[i]) / dx[i - 1])
        b = F(F(dy[i] * dx[i - 1]) / dx[i])
        d[i] = F(F(a + b) / F(dx[i - 1] + dx[i]))
    return d


def interp(x, y, xp):
    n = min(len(x), len(y))
    if n == 0:
        return F(0)
    if n == 1:
        return F(y[0])
    i = 0
    for k in range(n - 2, -1, -1):
        if x[k] < xp:
            i = k
            break
    slope = F(F(y[i + 1] - y[i]) / F(x[i + 1] - x[i]))
    intercept = F(y[i] - F(slope * x[i]))
    return F(F(slope * xp) + intercept)


class Panic(Exception):
    pass


def bisection(f, y0, xmin, xmax):
    tol = F(1.0e-6)
    if not xmin < xmax:
        raise Panic("assert xmin < xmax")
    x0, x1 = F(xmin), F(xmax)
    for _ in range(1000000):
        xmid = F(F(x0 + x1) / F(2))
        y = f(xmid)
        if abs(F(y - y0)) < tol:
            return xmid
        if abs(F(xmid - xmin)) < tol or abs(F(xmid - xmax)) < tol:
            raise Panic("bisection ended at a bound")
        if y < y0:
            x0 = xmid
        else:
            x1 = xmid
    raise Panic("bisection failed")


def bisect_array(f, roots, ytgt, lo, hi, xmin, xmax):
    n = hi - lo
    if n == 0:
        return
    if n == 1:
        roots[lo] = bisection(f, ytgt[lo], xmin, xmax)
        return
    mid = lo + n // 2
    bisect_array(f, roots, ytgt, mid, mid + 1, xmin, xmax)
    xm = roots[mid]
    bisect_array(f, roots, ytgt, lo, mid, xmin, xm)
    bisect_array(f, roots, ytgt, mid + 1, hi, xm, xmax)


def step(betas, momentum, round_trips, dhist, num_sweeps, num_chains, alpha, m):
    """-> (status, betas, momentum, tau, err); status 0 updated, 1 insufficient
    round trips (betas and momentum unchanged); raises Panic where the reference panics."""
    beta = [F(b) for b in betas]
    mom = [F(b) for b in momentum]
    alpha, m = F(alpha), F(m)
    nt = len(beta)
    difs = [F(beta[i + 1] - beta[i]) for i in range(nt - 1)]
    w = [F(0)] * nt
    w[0] = F(difs[0] / F(2))
    for i in range(1, nt - 1):
        w[i] = F(F(difs[i - 1] + difs[i]) / F(2))
    w[nt - 1] = F(difs[nt - 2] / F(2))
    taus, ddifs = [], []
    for rts, h in zip(round_trips, dhist):
        rt_per_rep = F(F(int(rts)) / F(num_chains * nt))
        taus.append(F(0) if rts == 0 else F(F(num_sweeps) / rt_per_rep))
        a = [F(int(h[t][0]) + 1) for t in range(nt)]
        b = [F(int(h[t][1]) + 1) for t in range(nt)]
        probs = [F(b[t] / F(a[t] + b[t])) for t in range(nt)]
        ddifs.append(finite_differences(beta, probs))
    sum_tau = nd_sum(taus)
    wdd = [F(0)] * nt
    for tau, d in zip(taus, ddifs):
        wdd = [F(wdd[t] + F(tau * d[t])) for t in range(nt)]
    wdd = [F(x / sum_tau) for x in wdd]
    eta = []
    for t in range(nt):
        v = F(wdd[t] / w[t])
        v = F(0) if (np.isnan(v) or v < 0) else v
        eta.append(F(np.sqrt(v)))
    eta_w = [F(F(F(eta[t] + eta[t + 1]) / F(2)) * difs[t]) for t in range(nt - 1)]
    z = nd_sum(eta_w)
    if z < F(np.finfo(np.float32).eps):
        return 1, list(beta), list(mom), taus, None
    cdf, acc = [], F(0)
    for t in range(nt - 1):
        cdf.append(acc)
        acc = F(acc + F(eta_w[t] / z))
    cdf.append(F(1))
    bmin, bmax = beta[0], beta[-1]

    def f(x):
        return interp(beta, cdf, F(bmin + F(x * F(bmax - bmin))))

    xd = [F(0)] * nt
    xd[-1] = F(1)
    tgt = [F(0)] + [F(i / (nt - 1)) for i in range(1, nt - 1)]
    bisect_array(f, xd, tgt, 1, nt - 1, F(0), F(1))
    calc = [F(F(x * F(bmax - bmin)) + bmin) for x in xd]
    mom = [expf(F(F(m * logf(bp)) + F(F(F(1) - m) * logf(b1)))) for bp, b1 in zip(mom, calc)]
    out = list(calc)
    err = F(0)
    for t in range(1, nt - 1):
        b = expf(F(F(alpha * logf(mom[t])) + F(F(F(1) - alpha) * logf(beta[t]))))
        err = F(err + F(abs(F(log10f(out[t]) - log10f(beta[t])))))
        out[t] = b
    return 0, out, mom, taus, F(err / F(nt))
