"""The reference's own acceptance criteria for its shipped example runs
(README.spp:101-105: the sinusoidal initial field of pfield.f, 20 steps, no
forcing): the turbulent kinetic energy does not increase, the first two rms
velocities are identical, and so are the first two Taylor microscales.  With
zero shifts the field on the grid also has pcheck.f's exact values, checked
through the stage-1 velmax and the velocity-gradient moments.
Checked on the device path, with the device field compared to the same
field built from pfield.f's formula and transformed by the oracle."""
import numpy as np
import pytest


def sinusoidal_ycyl(o, au=1.0, av=1.0):
    """pfield.f's field on the grid, transformed (numpy FFT, 1/n^3), kept in
    the cylinder columns: an independent construction of the modes."""
    n = o.n
    x = 2 * np.pi * np.arange(n) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    aw = -(au + av)
    phys = [au * np.sin(X) * np.cos(Y) * np.cos(Z), av * np.cos(X) * np.sin(Y) * np.cos(Z),
            aw * np.cos(X) * np.cos(Y) * np.sin(Z)]
    geo = o.geometry()
    kx = np.repeat(np.arange(len(geo["colstart"]) - 1), np.diff(geo["colstart"]))
    out = np.zeros(o.state_shape(), complex)
    for v in range(3):
        F = np.fft.fftn(phys[v]) / n ** 3           # F[kx, ky, kz]
        out[v] = F[kx[:, None], np.arange(n)[None, :], geo["az"][:, None]]
    out[np.abs(out) < 1e-14] = 0
    return out


def grid_checks(n, au=1.0, av=1.0):
    """pcheck.f's exact values on the grid x = (i-1) 2 pi/n: the stage-1
    velmax n max(|u|+|v|+|w|) (unit beta, zero shifts) and the raw moments
    1..8 of du/dx = au cos x cos y cos z and dw/dz = aw cos x cos y cos z."""
    x = 2 * np.pi * np.arange(n) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    aw = -(au + av)
    speed = (np.abs(au * np.sin(X) * np.cos(Y) * np.cos(Z)) + np.abs(av * np.cos(X) * np.sin(Y) * np.cos(Z))
             + np.abs(aw * np.cos(X) * np.cos(Y) * np.sin(Z)))
    ccc = np.cos(X) * np.cos(Y) * np.cos(Z)
    mom = lambda a: np.array([np.mean((a * ccc) ** m) for m in range(1, 9)])
    return n * speed.max(), mom(au), mom(aw)


def check_grid(velmax, moments, n, rtol):
    vm, mx, mz = grid_checks(n)
    np.testing.assert_allclose(velmax, vm, rtol=rtol)
    # odd moments vanish: compare against the scale of the even ones
    np.testing.assert_allclose(moments[0], mx, rtol=rtol, atol=rtol * mx[1])
    np.testing.assert_allclose(moments[1], mz, rtol=rtol, atol=rtol * mz[1] * 16)


def check_criteria(tke, scales):
    """README.spp:101-105 on a run's history: tke never increases; the first
    two rms velocities and the first two Taylor microscales agree."""
    assert np.all(np.diff(tke) <= 1e-12 * tke[0])
    assert tke[-1] < tke[0]
    np.testing.assert_allclose(scales["rms"][0], scales["rms"][1], rtol=1e-4)
    np.testing.assert_allclose(scales["taak"][0, 0], scales["taak"][1, 1], rtol=1e-4)


# (cfl, dt, kshift): fixed dt with shifts drawn each step, and the Courant
# controlled dt with kshift 4 of the shipped inputs (dir_runs*/input)
CASES = [(-1.0, 0.01, 1), (0.5, 0.0, 4)]


@pytest.mark.parametrize("cfl,dt,kshift", CASES)
def test_oracle_sinusoidal_criteria(oracle_mod, cfl, dt, kshift):
    n, nu = 32, 0.01
    o = oracle_mod.Oracle(n, nu, cfl=cfl, dt=dt, kshift=kshift)
    o.set_state(sinusoidal_ycyl(o))
    moments = o.gradient_moments()
    # the exact rms of pfield's field: au/sqrt(8), av/sqrt(8), 2/sqrt(8)
    np.testing.assert_allclose(o.spectra_scales()[3]["rms"], np.array([1, 1, 2]) / np.sqrt(8), rtol=1e-12)
    tke = [o.spectra()[3]["tke"]]
    for i in range(20):
        assert o.step() == 0
        if i == 0 and kshift == 4:
            check_grid(o.scalars()["velmax"], moments, n, 1e-12)
        tke.append(o.spectra()[3]["tke"])
    check_criteria(tke, o.spectra_scales()[3])
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("cfl,dt,kshift", CASES)
def test_sinusoidal_field_and_reference_criteria(oracle_mod, gpu_mod, prec, cfl, dt, kshift):
    n, nu = 32, 0.01
    o = oracle_mod.Oracle(n, nu, cfl=cfl, dt=dt, kshift=kshift)
    ref = sinusoidal_ycyl(o)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=cfl, dt=dt, kshift=kshift)
    s.field_sinusoidal(1.0, 1.0)
    np.testing.assert_allclose(s.get_state(gpu_mod.FIELD_UN), ref, rtol=0, atol=1e-7 if prec == 0 else 1e-15)
    o.set_state(ref)
    moments = s.gradient_moments()
    tke = [s.spectra()[3]["tke"]]
    for i in range(20):
        info = s.step()
        assert info["status"] == 0
        if i == 0 and kshift == 4:
            check_grid(info["velmax"], moments, n, 2e-6 if prec == 0 else 1e-12)
        o.step()
        tke.append(s.spectra()[3]["tke"])
    check_criteria(tke, s.spectra_scales()[3])
    # the device run follows the oracle
    _, un_o = o.get_state()
    un_g = s.get_state(gpu_mod.FIELD_UN)
    assert np.linalg.norm(un_g - un_o) / np.linalg.norm(un_o) < (2e-5 if prec == 0 else 1e-11)
    o.close()
    s.close()
