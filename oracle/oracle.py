"""ctypes binding of the CPU FP64 oracle (liboracle.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product library never
imports this module.

The oracle restates the PSDNS RK2 time step (timestep_module.f:70-481 and the
routines it calls) in FP64 C.  Parity status: pinned only by the reference's
own shipped checks (README.spp:101-105 eulstat criteria and pcheck.f's exact
grid values for the pfield.f sinusoidal field, tests/test_reference_criteria.py),
otherwise unpinned at the FFT boundary (the reference's FFTW is not vendored,
and the reference ships no golden vectors); the oracle FFT is cross-checked
against numpy.fft by the tests.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_destroy.argtypes = [vp]
        L.orc_kxn.argtypes = [vp]
        L.orc_xz_tot.argtypes = [vp]
        L.orc_geometry.argtypes = [vp, ip, ip, ip, ip]
        L.orc_set_state.argtypes = [vp, dp]
        L.orc_get_state.argtypes = [vp, dp, dp]
        L.orc_get_scalars.argtypes = [vp, dp]
        L.orc_step.argtypes = [vp]
        L.orc_stage.argtypes = [vp, ctypes.c_int]
        L.orc_set_rkmethod.argtypes = [vp, ctypes.c_int]
        L.orc_set_shifts.argtypes = [vp, dp]
        L.orc_itransform_only.argtypes = [vp, ctypes.c_int, dp, dp]
        L.orc_fft.argtypes = [dp, ctypes.c_int, ctypes.c_int]
        L.orc_field_init.argtypes = [vp, ctypes.c_int, dp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_set_forcing.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int]
        L.orc_get_forcing.argtypes = [vp, dp, dp]
        L.orc_rann2.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_spectra.argtypes = [vp, ctypes.c_int, dp, dp, dp, dp]
        L.orc_particles_set.argtypes = [vp, ctypes.c_long, dp]
        L.orc_particles_get.argtypes = [vp, dp, dp]
        L.orc_transfer_spectrum.argtypes = [vp, dp, dp]
        L.orc_spectra_scales.argtypes = [vp, ctypes.c_int, dp, dp, dp, dp]
        L.orc_particles_init.argtypes = [vp, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        L.orc_gradient_moments.argtypes = [vp, ctypes.c_int, dp, dp]
        L.orc_set_scalar.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def fft(x, sign):
    """Unnormalised complex FFT of a 1-D array (sign -1 forward, +1 backward)."""
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().orc_fft(_dp(a.view(np.float64)), a.size, int(sign))
    return a


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


def scales_dict(st):
    """The 55 scale statistics of sptr (psdns_gpu_spectra_scales order)."""
    return {"corr": st[0:6], "lijk": st[6:24].reshape(6, 3), "rms": st[24:27], "raak": st[27:30],
            "ett": st[30:33], "tmij": st[33:42].reshape(3, 3), "grdiss": st[42],
            "taak": st[43:52].reshape(3, 3), "tmre": st[52:55]}


class Oracle:
    """One periodic box advanced by the FP64 restatement of the RK2 step."""

    def __init__(self, n, viscos, cfl=-1.0, dt=0.005, kshift=1, seed_input=122929298, ksran=1,
                 beta=(1.0, 1.0, 1.0), rkmethod=2):
        self.n = n
        self.nc = 0
        self._c = lib().orc_create(n, viscos, cfl, dt, kshift, seed_input, ksran, *beta)
        self.kxn = lib().orc_kxn(self._c)
        self.xz_tot = lib().orc_xz_tot(self._c)
        if rkmethod != 2:
            assert lib().orc_set_rkmethod(self._c, int(rkmethod)) == 0, "rkmethod must be 2 or 4 (4: no scalar)"

    def close(self):
        if self._c:
            lib().orc_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def geometry(self):
        cut = np.zeros(self.kxn, np.int32)
        col = np.zeros(self.kxn + 1, np.int32)
        kym = np.zeros(self.xz_tot, np.int32)
        az = np.zeros(self.xz_tot, np.int32)
        lib().orc_geometry(self._c, _ip(cut), _ip(col), _ip(kym), _ip(az))
        return {"cut": cut, "colstart": col, "kymax": kym, "az": az}

    def set_scalar(self, pr=1.0, grad=(0.0, 1.0, 0.0)):
        """One passive scalar (nc = 1): Schmidt number pr, mean gradient grad.
        The state grows to 4 variables; the scalar starts at zero."""
        lib().orc_set_scalar(self._c, 1, float(pr), *[float(g) for g in grad])
        self.nc = 1

    def state_shape(self):
        return (3 + self.nc, self.xz_tot, self.n)

    def field_init(self, seed):
        """Velocity of field.f (3 variables); a scalar is left at zero."""
        out = np.zeros(self.state_shape(), np.complex128)
        lib().orc_field_init(self._c, int(seed), _dp(out[:3].view(np.float64)))
        return out

    def set_state(self, un):
        a = np.ascontiguousarray(un, dtype=np.complex128)
        assert a.shape == self.state_shape()
        lib().orc_set_state(self._c, _dp(a.view(np.float64)))

    def get_state(self):
        u = np.zeros(self.state_shape(), np.complex128)
        un = np.zeros(self.state_shape(), np.complex128)
        lib().orc_get_state(self._c, _dp(u.view(np.float64)), _dp(un.view(np.float64)))
        return u, un

    def scalars(self):
        out = np.zeros(11, np.float64)
        lib().orc_get_scalars(self._c, _dp(out))
        return {"dt": out[0], "time": out[1], "velmax": out[2], "dt2": out[3],
                "gsh": out[4:10].reshape(2, 3).T.copy(), "status": int(out[10])}

    def step(self):
        return lib().orc_step(self._c)

    def set_shifts(self, gsh):
        g = np.ascontiguousarray(gsh, dtype=np.float64).reshape(3, 2)
        lib().orc_set_shifts(self._c, _dp(g))

    def stage(self, kstep):
        return lib().orc_stage(self._c, int(kstep))

    def set_forcing(self, kforce, tforce, epsfor, tfiuo=0.0, kranf1=5, kranf2=5):
        """Eswaran-Pope forcing (force.f) with the reference's RNG sequences."""
        lib().orc_set_forcing(self._c, kforce, tforce, epsfor, tfiuo, kranf1, kranf2)
        bmin = 1.0
        self.kfor = int(kforce / bmin + 1.5)
        self.k2fo = 2 * self.kfor - 1

    def forcing(self):
        """(for(kfor,k2fo,k2fo,3) as a Fortran-ordered complex array, efkz[kfor,3])."""
        nf = self.kfor * self.k2fo * self.k2fo * 3
        tab = np.zeros(nf, np.complex128)
        ef = np.zeros(3 * self.kfor, np.float64)
        lib().orc_get_forcing(self._c, _dp(tab.view(np.float64)), _dp(ef))
        return tab.reshape(3, self.k2fo, self.k2fo, self.kfor), ef.reshape(self.kfor, 3)

    def spectra(self, which=1):
        """sptr.f restated: (ek[n], dk[n], eijk[n,6], stats dict) of un (which=1) or u."""
        n = self.n
        ek = np.zeros(n); dk = np.zeros(n); e6 = np.zeros(n * 6); st = np.zeros(7)
        lib().orc_spectra(self._c, int(which), _dp(ek), _dp(dk), _dp(e6), _dp(st))
        return ek, dk, e6.reshape(n, 6), dict(zip(["tke", "eps", "skew", "klen", "kvel", "ktime", "ekl"], st))

    def particles_set(self, pos):
        """pos: (np, 3) positions in grid units (pp(np,1:3))."""
        flat = np.ascontiguousarray(np.asarray(pos, np.float64).T)
        self._np = flat.shape[1]
        lib().orc_particles_set(self._c, self._np, _dp(flat))

    def particles_init(self, nop, pstart=0, kipran=11):
        """partin.f: positions made at the first particle phase (pstart 0:
        nop uniform random, -1: a lattice of nop^3 nodes)."""
        lib().orc_particles_init(self._c, int(nop), int(pstart), int(kipran))
        self._np = int(nop) if pstart == 0 else int(nop) ** 3

    def particles_get(self):
        pos = np.zeros((3, self._np)); vel = np.zeros((3, self._np))
        lib().orc_particles_get(self._c, _dp(pos), _dp(vel))
        return pos.T.copy(), vel.T.copy()

    def rann2(self, seq, n):
        x = np.zeros(n, np.float64)
        lib().orc_rann2(self._c, int(seq), _dp(x), int(n))
        return x

    def transfer_spectrum(self, gsh=(0.0, 0.0, 0.0)):
        """trfsp.f: T(k), k = 1..n/2, of u (convective term) against un."""
        g = np.ascontiguousarray(gsh, dtype=np.float64)
        tk = np.zeros(self.n // 2)
        lib().orc_transfer_spectrum(self._c, _dp(g), _dp(tk))
        return tk

    def spectra_scales(self, which=1):
        """sptr.f one-dimensional spectra (xr, yr, zr: [6, n/2+1]) and the
        scale statistics (dict of arrays)."""
        nh = self.n // 2 + 1
        xr = np.zeros(6 * nh); yr = np.zeros(6 * nh); zr = np.zeros(6 * nh); st = np.zeros(55)
        lib().orc_spectra_scales(self._c, int(which), _dp(xr), _dp(yr), _dp(zr), _dp(st))
        return xr.reshape(6, nh), yr.reshape(6, nh), zr.reshape(6, nh), scales_dict(st)

    def gradient_moments(self, which=1, gsh=(0.0, 0.0, 0.0)):
        """vgmomt.f: (moments 1..8 of du/dx, of dw/dz) on the grid shifted by gsh."""
        g = np.ascontiguousarray(gsh, dtype=np.float64)
        out = np.zeros(16, np.float64)
        lib().orc_gradient_moments(self._c, int(which), _dp(g), _dp(out))
        return out[:8].copy(), out[8:].copy()

    def itransform(self, ucyl, kstep=1):
        a = np.ascontiguousarray(ucyl, dtype=np.complex128)
        p = np.zeros((3, self.n, self.n, self.n), np.float64)
        lib().orc_itransform_only(self._c, int(kstep), _dp(a.view(np.float64)), _dp(p))
        return p
