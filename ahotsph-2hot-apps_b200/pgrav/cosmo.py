"""Background cosmology of the cosmological leapfrog (nlnhost.h nln_cosmo_*).

The reference's CosmoIntegrate (nln/integrate.c:82-135) takes a(t) and the
integrals kick(t0, t1) = int dt/a and drift(t0, t1) = int dt/a^2 from the
cosmology object of the 2hot support library; Cosmology integrates the same
Friedmann model (matter, radiation, curvature, a cosmological constant and
a w0 + wa (1 - a) dark-energy fluid) in the run's time unit.
"""
import ctypes

from .host import lib as _hostlib


class CosmoParams(ctypes.Structure):
    _fields_ = [("H0", ctypes.c_double), ("Omega_m", ctypes.c_double),
                ("Omega_r", ctypes.c_double), ("Omega_lambda", ctypes.c_double),
                ("Omega_de", ctypes.c_double), ("w0", ctypes.c_double), ("wa", ctypes.c_double)]


_bound = False


def _lib():
    global _bound
    L = _hostlib()
    if not _bound:
        vp, d = ctypes.c_void_p, ctypes.c_double
        L.nln_cosmo_new.argtypes = [ctypes.POINTER(CosmoParams)]
        L.nln_cosmo_new.restype = vp
        L.nln_cosmo_free.argtypes = [vp]
        for name in ("nln_cosmo_hubble", "nln_cosmo_t_at_a", "nln_cosmo_a_at_t"):
            getattr(L, name).argtypes = [vp, d]
            getattr(L, name).restype = d
        for name in ("nln_cosmo_kick", "nln_cosmo_drift"):
            getattr(L, name).argtypes = [vp, d, d]
            getattr(L, name).restype = d
        L.nln_cosmo_kdk.argtypes = [vp, d, d, d, d, ctypes.POINTER(ctypes.c_double)]
        _bound = True
    return L


class Cosmology:
    """H(a), t(a), a(t), kick and drift of a Friedmann model (t = 0 at a = 0).
    H0 is in the inverse of the run's time unit; the reference's default,
    0.0511365, is 100 km/s/Mpc in its units."""

    def __init__(self, H0=0.0511365, Omega_m=1.0, Omega_r=0.0, Omega_lambda=0.0, Omega_de=0.0,
                 w0=-1.0, wa=0.0):
        self.params = CosmoParams(H0, Omega_m, Omega_r, Omega_lambda, Omega_de, w0, wa)
        self._h = _lib().nln_cosmo_new(ctypes.byref(self.params))
        if not self._h:
            raise ValueError("cosmology: H0 > 0 and some matter or radiation are required")

    def __del__(self):
        try:
            if self._h:
                _lib().nln_cosmo_free(self._h)
                self._h = None
        except Exception:
            pass

    def hubble(self, a):
        return _lib().nln_cosmo_hubble(self._h, float(a))

    def t_at_a(self, a):
        return _lib().nln_cosmo_t_at_a(self._h, float(a))

    def a_at_t(self, t):
        return _lib().nln_cosmo_a_at_t(self._h, float(t))

    def kick(self, t0, t1):
        return _lib().nln_cosmo_kick(self._h, float(t0), float(t1))

    def drift(self, t0, t1):
        return _lib().nln_cosmo_drift(self._h, float(t0), float(t1))

    def kdk(self, tpos, tvel, dt, dtv):
        """CosmoIntegrate's six factors (nlnhost.h nln_cosmo_kdk)."""
        out = (ctypes.c_double * 6)()
        _lib().nln_cosmo_kdk(self._h, float(tpos), float(tvel), float(dt), float(dtv), out)
        return list(out)
