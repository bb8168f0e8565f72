"""The CPU oracle pinned against the reference's published known-answer values.

Sources of the pinned numbers (reference paths):
* AGENTS.md:114-124         grating.ofd convergence table at lambda = 461 nm
* .github/workflows/ci.yml:231-266  rcwa_rect2d / rcwa_oblique / rcwa_metal smokes
* tests/test_rcwa_input.cpp:129-155, 688-770   Fresnel checks
* ci/check_rcwa_ofd_dispersion.py:47-72, 143   Drude film vs transfer matrix
"""
import cmath
import math

import numpy as np
import pytest

from oracle.rcwa_oracle import (C0, ContinuousXY, DiscontinuousX, DiscontinuousY, OfdSetup,
                                RcwaLayerSpec as L, RcwaPole, fourier1d, fourier2d, gamma_sqrt,
                                rcwa_run, toeplitz_dense)

GRATING = [L(1, 1, .5, 0), L(4, 1, .5, 2e-7), L(2.25, 2.25, .5, 0)]


@pytest.mark.parametrize("N,rte,rtm", [(5, 0.138130, 0.204841), (12, 0.138187, 0.206747),
                                       (20, 0.138193, 0.206805)])
def test_grating_convergence_table(N, rte, rtm):
    # frequency1 = 4.3e14 7.5e14 16 gives f = 4.3e14 + n*0.2e14; n = 11 is 461 nm
    s = OfdSetup(nHx=N, period_x=3e-7, layers=GRATING, freqs=[4.3e14 + 11 * 0.2e14])
    r = rcwa_run(s)[0]
    assert abs(r["lam"] - 461.2e-9) < 1e-10
    assert abs(r["R"][0] - rte) < 1e-6 and abs(r["R"][1] - rtm) < 1e-6
    assert np.all(np.abs(r["R"] + r["T"] - 1) < 1e-10)


def test_oblique_brewster():
    s = OfdSetup(nHx=3, period_x=3e-7, layers=[L(1, 1, .5, 0), L(2.25, 2.25, .5, 0)],
                 freqs=[5e14], theta=56.30993247)
    r = rcwa_run(s)[0]
    assert abs(r["R"][0] - 0.147929) < 1e-6
    assert r["R"][1] < 1e-8
    assert np.all(np.abs(r["R"] + r["T"] - 1) < 1e-10)


def test_metal_film():
    s = OfdSetup(nHx=3, period_x=3e-7,
                 layers=[L(1, 1, .5, 0), L(-17.74, -17.74, .5, 3e-8, .18, .18), L(2.25, 2.25, .5, 0)],
                 freqs=[4.9966e14])
    r = rcwa_run(s)[0]
    assert abs(r["R"][0] - 0.909420) < 1e-6 and abs(r["T"][0] - 0.084430) < 1e-6


def test_rect2d_c4_symmetry_and_energy():
    s = OfdSetup(nHx=3, period_x=5e-7, nHy=3, period_y=5e-7,
                 layers=[L(1, 1, .5, 0), L(2.25, 1, .6, 2e-7, 0, 0, .6), L(2.25, 2.25, .5, 0)],
                 freqs=[3.331e14, 4.835e14])
    for r in rcwa_run(s):
        assert (r["R"][0] - r["R"][1]) ** 2 < 1e-12 and (r["T"][0] - r["T"][1]) ** 2 < 1e-12
        assert np.all((r["R"] + r["T"] - 1) ** 2 < 1e-12)


def _fresnel(n1, n2, th):
    ci = math.cos(th)
    st = n1 * math.sin(th) / n2
    ct = cmath.sqrt(1 - st * st)
    rs = (n1 * ci - n2 * ct) / (n1 * ci + n2 * ct)
    rp = (n2 * ci - n1 * ct) / (n2 * ci + n1 * ct)
    return abs(rs) ** 2, abs(rp) ** 2


@pytest.mark.parametrize("theta", [0.0, 15.0, 30.0, 45.0, 60.0, 75.0])
def test_fresnel_angle_sweep(theta):
    s = OfdSetup(nHx=2, period_x=3e-7, layers=[L(1, 1, .5, 0), L(2.25, 2.25, .5, 0)],
                 freqs=[5e14], theta=theta, phi=30.0)
    r = rcwa_run(s)[0]
    rs, rp = _fresnel(1.0, 1.5, math.radians(theta))
    assert abs(r["R"][0] - rs) < 1e-10 and abs(r["R"][1] - rp) < 1e-10


def _film_rt(eps_film, d, lam, n1=1.0, n3=1.5):
    """Airy thin-film formula at normal incidence (transfer-matrix analytic)."""
    n2 = cmath.sqrt(eps_film)
    if n2.imag < 0:
        n2 = -n2
    r12 = (n1 - n2) / (n1 + n2)
    r23 = (n2 - n3) / (n2 + n3)
    t12 = 2 * n1 / (n1 + n2)
    t23 = 2 * n2 / (n2 + n3)
    b = 2 * math.pi / lam * n2 * d
    e1 = cmath.exp(1j * b)
    den = 1 + r12 * r23 * e1 * e1
    r = (r12 + r23 * e1 * e1) / den
    t = t12 * t23 * e1 / den
    return abs(r) ** 2, (n3 / n1) * abs(t) ** 2


def test_drude_film_vs_transfer_matrix():
    freqs = [4e14 + k * 0.5e14 for k in range(7)]
    poles = [RcwaPole(1, 1, 1.0, 1.36e16, 3.0e13, 0.0), RcwaPole(1, 2, 1.0, 1.36e16, 3.0e13, 0.0)]
    s = OfdSetup(nHx=2, period_x=5e-7, layers=[L(1, 1, .5, 0), L(1, 1, .5, 3e-8), L(2.25, 2.25, .5, 0)],
                 freqs=freqs, poles=poles)
    for r in rcwa_run(s):
        w = 2 * math.pi * r["freq"]
        eps = 1.0 + 1.36e16 ** 2 / complex(0.0 - w * w, -3.0e13 * w)
        R, T = _film_rt(eps, 3e-8, r["lam"])
        assert abs(r["R"][0] - R) < 1e-9 and abs(r["T"][0] - T) < 1e-9
        assert r["R"][0] + r["T"][0] < 1


def test_orders_sum_to_totals():
    s = OfdSetup(nHx=4, period_x=6e-7, layers=GRATING, freqs=[5e14], theta=20.0, phi=10.0)
    r = rcwa_run(s)[0]
    assert np.all(np.abs(r["REF"].sum(axis=1) - r["R"]) < 1e-10)
    assert np.all(np.abs(r["TRN"].sum(axis=1) - r["T"]) < 1e-10)


def test_fill_y_one_2d_equals_1d():
    lay1 = [L(1, 1, .5, 0), L(4, 1, .4, 1.5e-7), L(2.25, 2.25, .5, 0)]
    r1 = rcwa_run(OfdSetup(nHx=4, period_x=4e-7, layers=lay1, freqs=[5e14]))[0]
    r2 = rcwa_run(OfdSetup(nHx=4, period_x=4e-7, nHy=2, period_y=4e-7, layers=lay1, freqs=[5e14]))[0]
    assert np.all(np.abs(r1["R"] - r2["R"]) < 1e-7) and np.all(np.abs(r1["T"] - r2["T"]) < 1e-7)


def test_fourier_building_blocks():
    x = np.array([0.0, 0.3, 1.0])
    f = np.array([2.0 + 0.5j, 1.0])
    F = fourier1d(x, 1.0, f, 5)
    # F_0 is the cell average; F_m follows the closed form
    assert abs(F[2] - (0.3 * f[0] + 0.7 * f[1])) < 1e-15
    m = 1
    ref = sum(fc * (x1 - x0) * np.exp(-1j * m * math.pi * (x1 + x0)) * np.sinc(m * (x1 - x0))
              for fc, x0, x1 in zip(f, x[:-1], x[1:]))
    assert abs(F[3] - ref) < 1e-14
    T = toeplitz_dense(F)
    assert T.shape == (3, 3) and T[1, 0] == F[3] and T[0, 1] == F[1]
    eps = np.array([[4.0, 1.0], [1.0, 1.0]], dtype=complex)
    cx = cy = np.array([0.0, 0.5, 1.0])
    for opt in (ContinuousXY, DiscontinuousX, DiscontinuousY):
        Ff = fourier2d(cx, cy, eps, 3, 3, opt)
        assert Ff.shape == (9, 9)
    # uniform layer: every rule gives eps*I
    for opt in (ContinuousXY, DiscontinuousX, DiscontinuousY):
        Ff = fourier2d(cx, cy, np.full((2, 2), 2.5 + 0.1j), 3, 3, opt)
        assert np.allclose(Ff, (2.5 + 0.1j) * np.eye(9), atol=1e-14)


def test_gamma_sqrt_branches():
    g = gamma_sqrt(np.array([4.0, -4.0, -4.0 - 0j, 1 - 1j, -1 - 1j, -1 + 1j]))
    assert np.allclose(g[:2], [2.0, 2j])
    assert g[2].imag > 0
    assert g[3].real > 0 and g[3].imag < 0          # 4th quadrant: principal root
    assert g[4].real < 0 and g[4].imag > 0          # 3rd quadrant: negated root
    assert g[5].real > 0 and g[5].imag > 0


def test_circle_fourier_closed_form():
    # analytic circular-pillar coefficients: exact mean, conjugate symmetry of
    # a real profile, and convergence of uniform staircases towards them
    import oracle.rcwa_oracle as ro
    Lx, Ly, R, c = 4e-7, 5e-7, 1.3e-7, (2.1e-7, 2.4e-7)
    e1, e2, nx, ny = 4.0, 1.0, 4, 3
    F = ro.circle_fourier2d(Lx, Ly, R, c, e1, e2, nx, ny)
    assert abs(F[nx - 1, ny - 1] - (e2 + (e1 - e2) * np.pi * R * R / (Lx * Ly))) < 1e-15
    assert np.allclose(F, np.conj(F[::-1, ::-1]), atol=1e-15)
    errs = []
    for cells in (50, 200, 800):
        cx, cy, eps = ro.circle_staircase(Lx, Ly, R, c, e1, e2, cells)
        F2D = np.zeros_like(F)
        for i in range(cells):
            F2D += np.outer(ro.fourier1d(cx, Lx, eps[i, :], 2 * nx - 1),
                            ro.fourier1d([cy[i], cy[i + 1]], Ly, [1.0], 2 * ny - 1))
        errs.append(np.max(np.abs(F2D - F)) / (e1 - e2))
    assert errs[2] < 1e-4 and errs[2] < errs[1] < errs[0]
    # the block-Toeplitz convolution matrix of the Laurent rule
    T = ro.block_toeplitz_dense(F)
    assert T.shape == (nx * ny, nx * ny) and np.allclose(np.diag(T), F[nx - 1, ny - 1])
