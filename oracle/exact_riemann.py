"""Test infrastructure (the oracle), not part of the product: the exact solution of the 1-D Riemann problem of an ideal
gas, the check of every shock tube of the batched configuration.

Restates the reference's validation oracle python/fenice/exact.py:5-70 (Toro, "Riemann Solvers and Numerical Methods
for Fluid Dynamics", 3rd ed. 2009, ch. 4): Newton iteration on the star pressure from the two-rarefaction-free guess
p = (pL + pR)/2 with the pressure functions f_K and their derivatives (shock branch for p > p_K, rarefaction branch
otherwise), clamped at 1e-12 and stopped at a relative step of 1e-12; the star velocity (uL + uR + fR - fL)/2; then the
wave pattern sampled at s = (x - x0)/t (shock speeds, rarefaction heads / tails and the fan states). Vectorised over
the sample points here; the arithmetic per point is the reference's.
"""
import numpy as np


def star_state(left, right, gamma=1.4):
    """(p*, u*) of the Riemann problem left = (rho, u, p), right = (rho, u, p)."""
    rL, uL, pL = left
    rR, uR, pR = right
    g = gamma
    cL, cR = np.sqrt(g * pL / rL), np.sqrt(g * pR / rR)

    def f(p, rk, pk, ck):
        if p > pk:
            A, B = 2.0 / ((g + 1) * rk), (g - 1) / (g + 1) * pk
            q = np.sqrt(A / (p + B))
            return (p - pk) * q, q * (1 - (p - pk) / (2 * (p + B)))
        pr = p / pk
        return 2 * ck / (g - 1) * (pr ** ((g - 1) / (2 * g)) - 1), pr ** (-(g + 1) / (2 * g)) / (rk * ck)

    ps = 0.5 * (pL + pR)
    for _ in range(100):
        fl, dl = f(ps, rL, pL, cL)
        fr, dr = f(ps, rR, pR, cR)
        dp = -(fl + fr + uR - uL) / (dl + dr)
        ps = max(ps + dp, 1e-12)
        if abs(dp) < 1e-12 * ps:
            break
    fl, _ = f(ps, rL, pL, cL)
    fr, _ = f(ps, rR, pR, cR)
    return ps, 0.5 * (uL + uR + fr - fl)


def riemann(x, t, left, right, gamma=1.4, x0=0.5):
    """rho, u, p of the exact solution at the points x and time t > 0."""
    rL, uL, pL = left
    rR, uR, pR = right
    g = gamma
    cL, cR = np.sqrt(g * pL / rL), np.sqrt(g * pR / rR)
    ps, us = star_state(left, right, gamma)

    def star_rho(rk, pk):
        if ps > pk:
            r = ps / pk
            return rk * (r + (g - 1) / (g + 1)) / (r * (g - 1) / (g + 1) + 1)
        return rk * (ps / pk) ** (1 / g)

    rsL, rsR = star_rho(rL, pL), star_rho(rR, pR)
    s = (np.atleast_1d(np.asarray(x, dtype=np.float64)) - x0) / t
    rho, u, p = np.empty_like(s), np.empty_like(s), np.empty_like(s)
    lft = s < us
    # left of the contact
    if ps > pL:
        sl = uL - cL * np.sqrt((g + 1) / (2 * g) * ps / pL + (g - 1) / (2 * g))
        pre = lft & (s < sl)
        post = lft & ~(s < sl)
        fan = np.zeros_like(lft)
    else:
        shl, stl = uL - cL, us - cL * (ps / pL) ** ((g - 1) / (2 * g))
        pre = lft & (s < shl)
        post = lft & ~(s < shl) & (s > stl)
        fan = lft & ~(s < shl) & ~(s > stl)
    rho[pre], u[pre], p[pre] = rL, uL, pL
    rho[post], u[post], p[post] = rsL, us, ps
    if fan.any():
        sf = s[fan]
        uf = 2 / (g + 1) * (cL + (g - 1) / 2 * uL + sf)
        cf = 2 / (g + 1) * (cL + (g - 1) / 2 * (uL - sf))
        rho[fan], u[fan], p[fan] = rL * (cf / cL) ** (2 / (g - 1)), uf, pL * (cf / cL) ** (2 * g / (g - 1))
    # right of the contact
    rgt = ~lft
    if ps > pR:
        sr = uR + cR * np.sqrt((g + 1) / (2 * g) * ps / pR + (g - 1) / (2 * g))
        pre = rgt & (s > sr)
        post = rgt & ~(s > sr)
        fan = np.zeros_like(rgt)
    else:
        shr, strr = uR + cR, us + cR * (ps / pR) ** ((g - 1) / (2 * g))
        pre = rgt & (s > shr)
        post = rgt & ~(s > shr) & (s < strr)
        fan = rgt & ~(s > shr) & ~(s < strr)
    rho[pre], u[pre], p[pre] = rR, uR, pR
    rho[post], u[post], p[post] = rsR, us, ps
    if fan.any():
        sf = s[fan]
        uf = 2 / (g + 1) * (-cR + (g - 1) / 2 * uR + sf)
        cf = 2 / (g + 1) * (cR - (g - 1) / 2 * (uR - sf))
        rho[fan], u[fan], p[fan] = rR * (cf / cR) ** (2 / (g - 1)), uf, pR * (cf / cR) ** (2 * g / (g - 1))
    return rho, u, p
