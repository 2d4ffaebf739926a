"""Seeded synthetic particle sets (the inputs every benchmark and test uses).

* Plummer sphere: inverse-CDF radius r = a / sqrt(U^(-2/3) - 1), redrawn
  beyond rmax, isotropic angles.
* Hernquist sphere: M(<r) = M r^2/(r+a)^2, so r = a sqrt(U)/(1 - sqrt(U)),
  redrawn beyond rmax.
* Periodic box: an n^3 grid in a unit box displaced by a Gaussian random
  field.  The displacement is the Zel'dovich (curl-free) field of a density
  field with power spectrum P(k) proportional to k^slope, rescaled to the
  requested rms displacement (3-D rms, in units of the grid spacing), then
  wrapped into [0, 1).
"""
import numpy as np


def _isotropic(rng, r):
    n = len(r)
    cth = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    sth = np.sqrt(1.0 - cth * cth)
    return np.stack([r * sth * np.cos(phi), r * sth * np.sin(phi), r * cth], axis=1)


def _radii(rng, n, inv_cdf, rmax):
    out = np.empty(0)
    while len(out) < n:
        u = rng.uniform(0.0, 1.0, 2 * (n - len(out)) + 16)
        u = u[(u > 0.0) & (u < 1.0)]
        r = inv_cdf(u)
        out = np.concatenate([out, r[r <= rmax]])
    return out[:n]


def plummer(n, seed=123, a=1.0, rmax=20.0, total_mass=1.0):
    """Positions (n,3) float32 and equal masses (n,) float32 of a Plummer sphere."""
    rng = np.random.default_rng(seed)
    r = _radii(rng, n, lambda u: a / np.sqrt(u ** (-2.0 / 3.0) - 1.0), rmax * a)
    pos = _isotropic(rng, r)
    return pos.astype(np.float32), np.full(n, total_mass / n, dtype=np.float32)


def hernquist(n, seed=123, a=1.0, rmax=20.0, total_mass=1.0):
    rng = np.random.default_rng(seed)
    r = _radii(rng, n, lambda u: a * np.sqrt(u) / (1.0 - np.sqrt(u)), rmax * a)
    pos = _isotropic(rng, r)
    return pos.astype(np.float32), np.full(n, total_mass / n, dtype=np.float32)


def grf_box(n1d, seed=123, slope=-2.5, rms_disp=0.25, total_mass=1.0):
    """n1d^3 particles in the unit box, Zel'dovich-displaced by a GRF."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n1d) * n1d           # integer wavenumbers
    kz = np.fft.rfftfreq(n1d) * n1d
    KX, KY, KZ = np.meshgrid(k, k, kz, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    k2[0, 0, 0] = 1.0
    amp = np.sqrt(k2 ** (slope / 2.0))
    amp[0, 0, 0] = 0.0
    white = rng.standard_normal((n1d, n1d, n1d))
    delta_k = np.fft.rfftn(white) * amp
    del white
    spacing = 1.0 / n1d
    disp = np.empty((n1d, n1d, n1d, 3), dtype=np.float64)
    for d, K in enumerate((KX, KY, KZ)):
        # psi_k = i k / k^2 delta_k  (so that div psi = -delta)
        disp[..., d] = np.fft.irfftn(1j * K / k2 * delta_k, s=(n1d, n1d, n1d), axes=(0, 1, 2))
    del delta_k
    rms = np.sqrt(np.mean(np.sum(disp * disp, axis=-1)))
    disp *= rms_disp * spacing / rms
    g = (np.arange(n1d) + 0.5) * spacing
    GX, GY, GZ = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([GX, GY, GZ], axis=-1) + disp
    pos = np.mod(pos, 1.0).reshape(-1, 3).astype(np.float32)
    pos[pos >= 1.0] = 0.0  # float rounding of values just below 1
    n = n1d ** 3
    return pos, np.full(n, total_mass / n, dtype=np.float32)


def uneven_batch(nsys=1024, seed=123, nmin=512, nmax=65536, eps_frac=0.01):
    """Independent isolated systems with log-uniform N in [nmin, nmax]; even
    systems Plummer, odd Hernquist (a=1), masses 1/N per system."""
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(nmin), np.log(nmax), nsys))).astype(np.int64)
    systems = []
    for s, n in enumerate(sizes):
        gen = plummer if s % 2 == 0 else hernquist
        systems.append(gen(int(n), seed=seed * 7919 + s))
    return systems
