"""Stability of the time step with dispersive cells, as the reference's
updates define it.

One Yee mode of a homogeneous medium advanced by the reference's operator
sequence (YeeUpdate on D, the material update, YeeUpdate on B; one-pole
DrudeUpdate of DispersiveMaterials.hpp:979-998, two-pole Lorentz as the
build's multi-pole extension of :710-735) is a linear map of (D, P, J, H);
its spectral radius must not exceed 1 for any mode. In grid units (c = eps0
= mu0 = 1, j = dt J) with s = 2 S sin(theta/2) the mode's curl symbol, S the
3D Courant number c dt sqrt(3)/dx:
  D' = D + s H;  P' = P + j;  E' = (D' - sum P') / eps_inf;
  Drude:   j' = (1-b)/(1+b) j + (wp dt)^2 E',      b = gamma dt / 2;
  Lorentz: j' = (1-g)/(1+g) j + (w0 dt)^2/(1+g) (d_eps E' - P'),  g = gamma dt;
  H' = H - s E'.
The Drude sphere workload (wp dt = 0.3, gamma dt = 0.01) is stable at
S = 0.98 and not at 0.99 (the highest mode grows by ~1.1 per step there: the
bound is 4 S^2 + (wp dt)^2 <= 4); the two-pole Lorentz workload is stable at
0.99 for every eps_inf of its blocks.
"""
import math

import numpy as np
import pytest


def _radius(s, drude=None, poles=(), eps=1.0):
    n = 2 + 2 * (1 if drude else len(poles))
    I = np.eye(n)
    D = I[0] + s * I[n - 1]
    rows = [D]
    if drude:
        w, b = drude
        P = I[1] + I[2]
        E = (D - P) / eps
        rows += [P, (1 - b) / (1 + b) * I[2] + w * w * E]
    else:
        Ps = [I[1 + 2 * q] + I[2 + 2 * q] for q in range(len(poles))]
        E = (D - sum(Ps)) / eps
        for q, (de, w0, g) in enumerate(poles):
            rows += [Ps[q], (1 - g) / (1 + g) * I[2 + 2 * q] + w0 * w0 / (1 + g) * (de * E - Ps[q])]
    rows.append(I[n - 1] - s * E)
    return float(max(abs(np.linalg.eigvals(np.vstack(rows)))))


def _worst(S, **kw):
    return max(_radius(s, **kw) for s in np.linspace(0.0, 2.0 * S, 2001))


def test_drude_sphere_is_stable_at_its_courant_number():
    from fdtd_b200 import problem as P
    p = P.config2(n=64, steps=2)
    S = P.C0 * p.dt * math.sqrt(3.0) / p.dx
    assert S == pytest.approx(0.98)
    assert _worst(S, drude=(0.3, 0.005)) <= 1.0 + 1e-9


def test_drude_sphere_would_grow_at_courant_099():
    # the bound 4 S^2 + (wp dt)^2 <= 4 of this update
    assert _worst(0.99, drude=(0.3, 0.005)) > 1.05
    assert _worst(math.sqrt(1.0 - 0.3 ** 2 / 4.0) - 1e-3, drude=(0.3, 0.005)) <= 1.0 + 1e-9


@pytest.mark.parametrize("eps", [1.0, 2.5, 6.0])
def test_two_pole_lorentz_is_stable_at_courant_099(eps):
    poles = [(1.5, 0.1, 0.005), (0.8, 0.25, 0.02)]
    assert _worst(0.99, poles=poles, eps=eps) <= 1.0 + 1e-9
