"""The background cosmology of the cosmological leapfrog (pgrav.cosmo,
nlnhost.h nln_cosmo_*) against closed forms -- Einstein-de Sitter, flat
Lambda-CDM, matter + radiation -- and direct quadrature.  CPU only."""
import numpy as np
import pytest
from scipy import integrate


def test_einstein_de_sitter_closed_forms():
    from pgrav.cosmo import Cosmology
    H0 = 0.0511365
    c = Cosmology(H0=H0, Omega_m=1.0)
    for a in (1e-3, 0.02, 0.5, 1.0, 3.0):
        t = 2.0 / (3.0 * H0) * a ** 1.5
        assert c.t_at_a(a) == pytest.approx(t, rel=1e-12)
        assert c.a_at_t(t) == pytest.approx(a, rel=1e-12)
    a0, a1 = 0.1, 0.13
    t0, t1 = c.t_at_a(a0), c.t_at_a(a1)
    # int dt/a = int da/(a^2 H), H = H0 a^-3/2
    assert c.kick(t0, t1) == pytest.approx(2.0 * (np.sqrt(a1) - np.sqrt(a0)) / H0, rel=1e-12)
    assert c.drift(t0, t1) == pytest.approx(2.0 * (1 / np.sqrt(a0) - 1 / np.sqrt(a1)) / H0,
                                            rel=1e-12)
    # backwards is the negative
    assert c.kick(t1, t0) == pytest.approx(-c.kick(t0, t1), rel=1e-14)


def test_flat_lambda_cdm_closed_forms():
    from pgrav.cosmo import Cosmology
    H0, Om, OL = 1.0, 0.3, 0.7
    c = Cosmology(H0=H0, Omega_m=Om, Omega_lambda=OL)
    for a in (1e-4, 0.1, 0.5, 1.0, 2.0):
        t = 2.0 / (3.0 * H0 * np.sqrt(OL)) * np.arcsinh(np.sqrt(OL / Om) * a ** 1.5)
        assert c.t_at_a(a) == pytest.approx(t, rel=1e-12)
        assert c.a_at_t(t) == pytest.approx(a, rel=1e-12)
        assert c.hubble(a) == pytest.approx(H0 * np.sqrt(Om * a ** -3 + OL), rel=1e-14)
    H = lambda a: H0 * np.sqrt(Om * a ** -3 + OL)
    a0, a1 = 0.4, 0.47
    t0, t1 = c.t_at_a(a0), c.t_at_a(a1)
    k = integrate.quad(lambda a: 1 / (a * a * H(a)), a0, a1, epsabs=0, epsrel=1e-13)[0]
    d = integrate.quad(lambda a: 1 / (a ** 3 * H(a)), a0, a1, epsabs=0, epsrel=1e-13)[0]
    assert c.kick(t0, t1) == pytest.approx(k, rel=1e-11)
    assert c.drift(t0, t1) == pytest.approx(d, rel=1e-11)


def test_matter_radiation_and_dark_energy():
    from pgrav.cosmo import Cosmology
    H0, Om, Or = 1.0, 0.3, 8e-5
    c = Cosmology(H0=H0, Omega_m=Om, Omega_r=Or, Omega_lambda=1 - Om - Or)
    for a in (1e-9, 1e-6, 1e-3):
        # radiation + matter dominate: t(a) in closed form
        t = 2.0 / (3.0 * H0 * Om ** 2) * ((Om * a - 2 * Or) * np.sqrt(Om * a + Or) + 2 * Or ** 1.5)
        assert c.t_at_a(a) == pytest.approx(t, rel=1e-6 if a > 1e-4 else 1e-9)
    # a w0-wa fluid: t(a) against direct quadrature of da / (a H)
    d = Cosmology(H0=H0, Omega_m=0.3, Omega_de=0.7, w0=-0.9, wa=0.2)
    H = lambda a: H0 * np.sqrt(0.3 * a ** -3 + 0.7 * a ** (-3 * (1 - 0.9 + 0.2)) * np.exp(-3 * 0.2 * (1 - a)))
    for a in (0.2, 1.0):
        t = integrate.quad(lambda x: 1 / (x * H(x)), 0, a, epsabs=0, epsrel=1e-13, limit=200)[0]
        assert d.t_at_a(a) == pytest.approx(t, rel=1e-10)
        assert d.a_at_t(t) == pytest.approx(a, rel=1e-12)


def test_kdk_factors():
    from pgrav.cosmo import Cosmology
    c = Cosmology(H0=0.0511365, Omega_m=0.3, Omega_lambda=0.7)
    tpos, dt = c.t_at_a(0.5), 0.3
    tvel = tpos - 0.5 * dt
    dtv = tpos + 0.5 * dt - tvel
    f = c.kdk(tpos, tvel, dt, dtv)
    a0 = c.a_at_t(tpos)
    assert f[0] == pytest.approx(a0 * a0 * c.kick(tvel, tpos), rel=1e-14)
    assert f[1] == pytest.approx(a0 * a0 * c.kick(tvel, tvel + dtv), rel=1e-14)
    assert f[2] == pytest.approx(c.drift(tpos, tpos + dt), rel=1e-14)
    assert f[3] == pytest.approx(1 / a0, rel=1e-14)
    assert f[4] == pytest.approx(c.a_at_t(tpos + dt), rel=1e-14)
    assert f[5] == pytest.approx(1 / a0 ** 2, rel=1e-14)
    with pytest.raises(ValueError):
        Cosmology(H0=0.0)
