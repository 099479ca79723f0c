"""Pins of the correlation functionals that the reference's tests leave
unpinned (VWN5, PW92 in both constant sets, PBE correlation): the oracle's
energies per particle against a second, independent restatement of the
published closed forms evaluated here in 40-digit arithmetic (mpmath).  The
oracle is C++ in complex-step form; this one is written from the papers'
equations with their published parameters:

  VWN5:  S. H. Vosko, L. Wilk, M. Nusair, Can. J. Phys. 58, 1200 (1980),
         their Pade-type closed form with the parameters of fit V for the
         paramagnetic, ferromagnetic and spin-stiffness curves, interpolated
         in zeta through the spin stiffness (libxc's LDA_C_VWN);
  PW92:  J. P. Perdew, Y. Wang, Phys. Rev. B 45, 13244 (1992), eqs. 8-10 and
         Table I (LDA_C_PW), and the same with the unrounded constants
         (LDA_C_PW_MOD, the one inside PBE);
  PBE-C: J. P. Perdew, K. Burke, M. Ernzerhof, Phys. Rev. Lett. 77, 3865
         (1996): PW92 plus the gradient term H(rs, zeta, t).

The oracle is in turn compared with the CUDA functionals in
tests/test_gpu_parity.py, so these pins reach the device path."""
import math

import numpy as np
import pytest

mp = pytest.importorskip("mpmath")

from oracle import oracle as O  # noqa: E402

mp.mp.dps = 40
PI = mp.pi


def f_zeta(z):
    return (mp.power(1 + z, mp.mpf(4) / 3) + mp.power(1 - z, mp.mpf(4) / 3) - 2) / (mp.power(2, mp.mpf(4) / 3) - 2)


def vwn_curve(x, A, x0, b, c):
    # A [ln(x^2/X) + 2b/Q atan(Q/(2x+b)) - b x0/X(x0) (ln((x-x0)^2/X) + 2(b+2x0)/Q atan(Q/(2x+b)))]
    X = lambda y: y * y + b * y + c  # noqa: E731
    Q = mp.sqrt(4 * c - b * b)
    at = mp.atan(Q / (2 * x + b))
    return A * (mp.log(x * x / X(x)) + 2 * b / Q * at
                - b * x0 / X(x0) * (mp.log((x - x0) ** 2 / X(x)) + 2 * (b + 2 * x0) / Q * at))


def eps_vwn5(rs, z):
    x = mp.sqrt(rs)
    eP = vwn_curve(x, mp.mpf("0.0310907"), mp.mpf("-0.10498"), mp.mpf("3.72744"), mp.mpf("12.9352"))
    eF = vwn_curve(x, mp.mpf("0.01554535"), mp.mpf("-0.32500"), mp.mpf("7.06042"), mp.mpf("18.0578"))
    aC = vwn_curve(x, -1 / (6 * PI * PI), mp.mpf("-0.0047584"), mp.mpf("1.13107"), mp.mpf("13.0045"))
    fpp0 = 4 / (9 * (mp.cbrt(2) - 1))
    f = f_zeta(z)
    return eP + aC * f / fpp0 * (1 - z ** 4) + (eF - eP) * f * z ** 4


def pw92_G(rs, A, a1, b1, b2, b3, b4):
    # eq. 10 with p = 1
    return -2 * A * (1 + a1 * rs) * mp.log(1 + 1 / (2 * A * (b1 * mp.sqrt(rs) + b2 * rs + b3 * rs ** mp.mpf(1.5)
                                                              + b4 * rs * rs)))


def eps_pw92(rs, z, mod):
    m = mp.mpf
    if mod:
        AP, AF, AA, fz20 = m("0.0310907"), m("0.01554535"), m("0.0168869"), 4 / (9 * (mp.cbrt(2) - 1))
    else:
        AP, AF, AA, fz20 = m("0.031091"), m("0.015545"), m("0.016887"), m("1.709921")
    ec0 = pw92_G(rs, AP, m("0.21370"), m("7.5957"), m("3.5876"), m("1.6382"), m("0.49294"))
    ec1 = pw92_G(rs, AF, m("0.20548"), m("14.1189"), m("6.1977"), m("3.3662"), m("0.62517"))
    mac = pw92_G(rs, AA, m("0.11125"), m("10.357"), m("3.6231"), m("0.88026"), m("0.49671"))  # -alpha_c
    f = f_zeta(z)
    # eq. 8
    return ec0 - mac * f / fz20 * (1 - z ** 4) + (ec1 - ec0) * f * z ** 4


def eps_pbe_c(rho, z, sigma):
    beta = mp.mpf("0.06672455060314922")
    gamma = (1 - mp.log(2)) / (PI * PI)
    rs = mp.cbrt(3 / (4 * PI * rho))
    ec = eps_pw92(rs, z, True)
    phi = (mp.power(1 + z, mp.mpf(2) / 3) + mp.power(1 - z, mp.mpf(2) / 3)) / 2
    kF = mp.cbrt(3 * PI * PI * rho)
    ks = mp.sqrt(4 * kF / PI)
    t2 = sigma / (2 * phi * ks * rho) ** 2
    A = beta / gamma / (mp.exp(-ec / (gamma * phi ** 3)) - 1)
    H = gamma * phi ** 3 * mp.log(1 + beta / gamma * t2 * (1 + A * t2) / (1 + A * t2 + A * A * t2 * t2))
    return ec + H


RS = (0.05, 0.3, 1.0, 2.0, 5.0, 12.0, 60.0)
ZETA = (0.0, 0.35, -0.8, 1.0)


def spin_densities(rs, z):
    rho = 3.0 / (4.0 * math.pi * rs ** 3)
    return rho, 0.5 * rho * (1 + z), 0.5 * rho * (1 - z)


@pytest.mark.parametrize("fid,ref", [(7, lambda rs, z: eps_vwn5(rs, z)),
                                     (12, lambda rs, z: eps_pw92(rs, z, False)),
                                     (13, lambda rs, z: eps_pw92(rs, z, True))])
def test_lda_correlation_matches_published_form(fid, ref):
    for rs in RS:
        for z in ZETA:
            rho, ra, rb = spin_densities(rs, z)
            e, _, _ = O.xc_eval(fid, 2, [ra, rb], [0.0, 0.0, 0.0])
            want = float(ref(mp.mpf(rs), mp.mpf(z)))
            assert e[0] == pytest.approx(want, rel=1e-12, abs=1e-15), (fid, rs, z, e[0], want)
            if z == 0.0:  # the unpolarised entry point agrees
                e1, _, _ = O.xc_eval(fid, 1, [rho], [0.0])
                assert e1[0] == pytest.approx(want, rel=1e-12)


def test_pbe_correlation_matches_published_form():
    rng = np.random.default_rng(11)
    for rs in RS:
        for z in ZETA:
            rho, ra, rb = spin_densities(rs, z)
            kF = (3 * math.pi ** 2 * rho) ** (1 / 3)
            for s_red in (0.0, 0.3, 1.5, 6.0):  # |grad rho| = s 2 kF rho, spin parts along one direction
                g = s_red * 2 * kF * rho
                u = rng.normal(size=3)
                u /= np.linalg.norm(u)
                ga, gb = 0.5 * (1 + z) * g * u, 0.5 * (1 - z) * g * u
                saa, sab, sbb = float(ga @ ga), float(ga @ gb), float(gb @ gb)
                e, _, _ = O.xc_eval(130, 2, [ra, rb], [saa, sab, sbb])
                want = float(eps_pbe_c(mp.mpf(rho), mp.mpf(z), mp.mpf(g) ** 2))
                assert e[0] == pytest.approx(want, rel=1e-11, abs=1e-15), (rs, z, s_red, e[0], want)
