"""Beam integration rules, restated from Strut's ``src/mojo/elements/beam_integration.mojo``.

Points are returned on xi in [0, 1] with weights halved, exactly as
``beam_integration_rule`` maps them (beam_integration.mojo:224-243).  Python floats are IEEE
doubles and the operations below are the same sequence as the Mojo source, so the values match
bit for bit.
"""
from __future__ import annotations

import math


def _legendre_polynomial_and_derivative(n: int, x: float):
    # beam_integration.mojo:21-44
    if n == 0:
        return (1.0, 0.0, 0.0)
    if n == 1:
        return (x, 1.0, 1.0)
    pnm2 = 1.0
    pnm1 = x
    for k in range(2, n + 1):
        kf = float(k)
        pk = ((2.0 * kf - 1.0) * x * pnm1 - (kf - 1.0) * pnm2) / kf
        pnm2 = pnm1
        pnm1 = pk
    pn = pnm1
    pn_minus_1 = pnm2
    denom = x * x - 1.0
    if abs(denom) <= 1.0e-18:
        x_off = x - 1.0e-12 if x >= 0.0 else x + 1.0e-12
        alt = _legendre_polynomial_and_derivative(n, x_off)
        return (pn, pn_minus_1, alt[2])
    dpn = float(n) * (x * pn - pn_minus_1) / denom
    return (pn, pn_minus_1, dpn)


def _sort_points(x, w):
    # insertion sort, beam_integration.mojo:47-60
    n = len(x)
    for i in range(1, n):
        kx, kw = x[i], w[i]
        j = i - 1
        while j >= 0 and x[j] > kx:
            x[j + 1] = x[j]
            w[j + 1] = w[j]
            j -= 1
        x[j + 1] = kx
        w[j + 1] = kw


def _fill_lobatto(n: int):
    # beam_integration.mojo:64-129
    if n < 2:
        raise ValueError("Lobatto integration requires num_int_pts >= 2")
    if n == 3:
        return [-1.0, 0.0, 1.0], [1.0 / 3.0, 4.0 / 3.0, 1.0 / 3.0]
    if n == 5:
        return (
            [-1.0, -0.6546536707079772, 0.0, 0.6546536707079772, 1.0],
            [0.1, 0.5444444444444444, 0.7111111111111111, 0.5444444444444444, 0.1],
        )
    x = [0.0] * n
    w = [0.0] * n
    m = n - 1
    nf = float(n)
    x[0] = -1.0
    x[n - 1] = 1.0
    w[0] = 2.0 / (nf * (nf - 1.0))
    w[n - 1] = w[0]
    pi = 3.141592653589793
    for i in range(1, n - 1):
        root = math.cos(pi * float(i) / float(n - 1))
        for _ in range(80):
            pm, _pm1, dpm = _legendre_polynomial_and_derivative(m, root)
            denom = 1.0 - root * root
            if abs(denom) <= 1.0e-18:
                break
            ddpm = (2.0 * root * dpm - float(m * (m + 1)) * pm) / denom
            if abs(ddpm) <= 1.0e-24:
                break
            delta = dpm / ddpm
            root -= delta
            if abs(delta) <= 1.0e-14:
                break
        x[i] = root
        pm_root = _legendre_polynomial_and_derivative(m, root)[0]
        pm2 = pm_root * pm_root
        if pm2 <= 0.0:
            raise ValueError("failed to compute Lobatto integration weights")
        w[i] = 2.0 / (nf * (nf - 1.0) * pm2)
    _sort_points(x, w)
    return x, w


def _fill_legendre(n: int):
    # beam_integration.mojo:132-175
    if n < 1:
        raise ValueError("Legendre integration requires num_int_pts >= 1")
    if n == 1:
        return [0.0], [2.0]
    x = [0.0] * n
    w = [0.0] * n
    m = (n + 1) // 2
    pi = 3.141592653589793
    for i in range(m):
        root = math.cos(pi * (float(i) + 0.75) / (float(n) + 0.5))
        dpn = 0.0
        for _ in range(80):
            pn, _p1, dpn = _legendre_polynomial_and_derivative(n, root)
            if abs(dpn) <= 1.0e-24:
                break
            delta = pn / dpn
            root -= delta
            if abs(delta) <= 1.0e-14:
                break
        one_minus = 1.0 - root * root
        if one_minus <= 1.0e-24:
            raise ValueError("failed to compute Legendre integration weights")
        weight = 2.0 / (one_minus * dpn * dpn)
        x[i] = -root
        w[i] = weight
        x[n - 1 - i] = root
        w[n - 1 - i] = weight
    _sort_points(x, w)
    return x, w


def _fill_radau(n: int):
    # beam_integration.mojo:178-221
    if n < 1:
        raise ValueError("Radau integration requires num_int_pts >= 1")
    if n == 1:
        return [-1.0], [2.0]
    x = [0.0] * n
    w = [0.0] * n
    n_sq = float(n * n)
    x[0] = -1.0
    w[0] = 2.0 / n_sq
    pi = 3.141592653589793
    for i in range(1, n):
        root = math.cos(float(2 * i - 1) * pi / float(2 * n - 1))
        for _ in range(100):
            pn = _legendre_polynomial_and_derivative(n, root)
            pnm1 = _legendre_polynomial_and_derivative(n - 1, root)
            f = pn[0] + pnm1[0]
            fp = pn[2] + pnm1[2]
            if abs(fp) <= 1.0e-24:
                break
            delta = f / fp
            root -= delta
            if abs(delta) <= 1.0e-14:
                break
        x[i] = root
        pnm1v = _legendre_polynomial_and_derivative(n - 1, root)[0]
        denom = n_sq * pnm1v * pnm1v
        if denom <= 1.0e-24:
            raise ValueError("failed to compute Radau integration weights")
        w[i] = (1.0 - root) / denom
    _sort_points(x, w)
    return x, w


def beam_integration_rule(integration: str, num_int_pts: int):
    """(xis, weights) on [0, 1] as Strut's beam_integration_rule returns them."""
    if integration == "Lobatto":
        x, w = _fill_lobatto(num_int_pts)
    elif integration == "Legendre":
        x, w = _fill_legendre(num_int_pts)
    elif integration == "Radau":
        x, w = _fill_radau(num_int_pts)
    else:
        raise ValueError(f"unsupported beam integration: {integration}")
    xis = [0.5 * (xi + 1.0) for xi in x]
    ws = [wi * 0.5 for wi in w]
    return xis, ws
