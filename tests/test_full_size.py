"""The 1024^3 box of the benchmark, checked through properties that need no
oracle run at that size: the reference's own checks of its example runs
(README.spp:101-105 with the pfield.f sinusoidal field: kinetic energy never
increases, the first two rms velocities and the first two Taylor microscales
agree) and pcheck.f's exact grid values of that field (stage-1 velmax with
zero shifts, moments of du/dx and dw/dz)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def exact_velmax(n, au=1.0, av=1.0):
    """n max over the grid of |u| + |v| + |w| for pfield.f's field, one z
    plane at a time."""
    x = 2 * np.pi * np.arange(n) / n
    s, c = np.sin(x), np.cos(x)
    aw = -(au + av)
    best = 0.0
    for k in range(n):
        f = (np.abs(au * np.outer(s, c) * c[k]) + np.abs(av * np.outer(c, s) * c[k])
             + np.abs(aw * np.outer(c, c) * s[k]))
        best = max(best, float(f.max()))
    return n * best


def exact_moments(n, a):
    """Raw moments 1..8 of a cos x cos y cos z on the grid (separable)."""
    c = np.cos(2 * np.pi * np.arange(n) / n)
    return np.array([a ** m * np.mean(c ** m) ** 3 for m in range(1, 9)])


@pytest.mark.parametrize("prec,rtol,vtol", [(0, 1e-5, 2e-6), (1, 1e-11, 1e-12)])
def test_sinusoidal_1024_reference_checks(gpu_mod, prec, rtol, vtol):
    n, nu, dt = 1024, 1e-3, 2e-3
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=-1.0, dt=dt, kshift=4, kforce=0.0)
    s.field_sinusoidal(1.0, 1.0)
    mx, mz = s.gradient_moments()
    for got, want in ((mx, exact_moments(n, 1.0)), (mz, exact_moments(n, -2.0))):
        scale = abs(want[1])
        np.testing.assert_allclose(got, want, rtol=rtol, atol=rtol * scale * 16)
    tke = [s.spectra()[3]["tke"]]
    # tke = <u^2 + v^2 + w^2>/2 = (1 + 1 + 4)/8/2 on the grid
    np.testing.assert_allclose(tke[0], 0.375, rtol=max(rtol, 1e-12))
    for i in range(3):
        info = s.step()
        assert info["status"] == 0
        if i == 0:
            np.testing.assert_allclose(info["velmax"], exact_velmax(n), rtol=vtol)
        tke.append(s.spectra()[3]["tke"])
    assert np.all(np.diff(tke) <= 1e-7 * tke[0])
    assert tke[-1] < tke[0]
    sc = s.spectra_scales()[3]
    np.testing.assert_allclose(sc["rms"][0], sc["rms"][1], rtol=1e-4)
    np.testing.assert_allclose(sc["taak"][0, 0], sc["taak"][1, 1], rtol=1e-4)
    s.close()
