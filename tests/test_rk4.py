"""RK4 (rkmethod = 4, -DRKFOUR: timestep_module.f:295-308 with
homogeneous/advanc_1.f .. advanc_4.f), the scheme of every shipped
dir_runs*/input.  The oracle restates advanc_1..4 as written (the
integrating factor of the whole step applied in the first sub-stage only,
the accumulator u1 copied into un and u at the end of advanc_4.f:149-161,
stages 3 and 4 on the shifts of stages 1 and 2, shifts.f:133-136); the
device follows the oracle to 1e-11 in FP64 and 2e-5 in FP32, and the
reference's own acceptance criteria (README.spp:101-105) hold for the
sinusoidal field under RK4 with the shipped cfl = 3.77 and kshift = 4.

As written, the scheme converges at first order in dt (halving dt halves
the error against a fine-dt run): checked on the oracle."""
import numpy as np
import pytest

from test_reference_criteria import check_criteria, sinusoidal_ycyl


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_oracle_rk4_order_as_written(oracle_mod):
    n, nu, T = 32, 0.01, 0.05
    errs = []
    for dt in (0.005, 0.0025):
        ref = oracle_mod.Oracle(n, nu, cfl=-1, dt=dt / 8, kshift=4, rkmethod=4)
        o = oracle_mod.Oracle(n, nu, cfl=-1, dt=dt, kshift=4, rkmethod=4)
        u0 = o.field_init(5)
        o.set_state(u0)
        ref.set_state(u0)
        for _ in range(int(round(T / dt))):
            assert o.step() == 0
        for _ in range(int(round(T / dt)) * 8):
            assert ref.step() == 0
        errs.append(rel(o.get_state()[1], ref.get_state()[1]))
        o.close()
        ref.close()
    assert 1.7 < errs[0] / errs[1] < 2.3, errs


def test_oracle_rk4_sinusoidal_criteria(oracle_mod):
    n, nu = 32, 0.0028
    o = oracle_mod.Oracle(n, nu, cfl=3.77, dt=0.0, kshift=4, rkmethod=4)
    o.set_state(sinusoidal_ycyl(o))
    tke = [o.spectra()[3]["tke"]]
    for _ in range(20):
        assert o.step() == 0
        tke.append(o.spectra()[3]["tke"])
    check_criteria(tke, o.spectra_scales()[3])
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,prec,cfl,kshift", [(32, 1, -1.0, 1), (64, 1, 3.77, 4), (32, 1, 3.77, 2), (64, 0, -1.0, 1)])
def test_rk4_device_against_oracle(oracle_mod, gpu_mod, n, prec, cfl, kshift):
    nu, dt = 0.01, 0.004
    o = oracle_mod.Oracle(n, nu, cfl=cfl, dt=dt if cfl < 0 else 0.0, kshift=kshift, rkmethod=4)
    un0 = o.field_init(1234)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=cfl, dt=dt if cfl < 0 else 0.0, kshift=kshift,
                       rkmethod=4)
    s.set_state(un0)
    for _ in range(5):
        assert o.step() == 0
        info = s.step()
        assert info["status"] == 0
        so = o.scalars()
        assert abs(info["dt"] - so["dt"]) <= (1e-12 if prec else 1e-5) * so["dt"]
    u_o, un_o = o.get_state()
    tol = 1e-11 if prec else 2e-5
    assert rel(s.get_state(gpu_mod.FIELD_UN), un_o) < tol
    assert rel(s.get_state(gpu_mod.FIELD_U), u_o) < tol
    o.close()
    s.close()


@pytest.mark.gpu
def test_rk4_forced_device_against_oracle(oracle_mod, gpu_mod):
    n, nu, dt = 32, 0.02, 0.004
    kforce, tforce = 2.99, 0.5
    epsfor = 0.1 / (4.0 * (4.0 * np.pi / 3.0) * kforce ** 3)
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=dt, kshift=1, rkmethod=4)
    o.set_forcing(kforce, tforce, epsfor, 0.0)
    un0 = o.field_init(77)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=nu, cfl=-1, dt=dt, kshift=1, kforce=kforce,
                       tforce=tforce, epsfor=epsfor, tfiuo=0.0, rkmethod=4)
    s.set_state(un0)
    for _ in range(3):
        o.step()
        s.step()
    assert rel(s.get_state(gpu_mod.FIELD_UN), o.get_state()[1]) < 1e-11
    o.close()
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_rk4_shipped_case_reference_criteria(oracle_mod, gpu_mod, prec):
    """dir_runs1/input: rkmethod 4, kshift 4, cfl 3.77, unforced, nc 0, the
    sinusoidal field (viscosity 0.0028; 32^3 here)."""
    n, nu = 32, 0.0028
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=3.77, dt=0.0, kshift=4, rkmethod=4)
    s.field_sinusoidal(1.0, 1.0)
    o = oracle_mod.Oracle(n, nu, cfl=3.77, dt=0.0, kshift=4, rkmethod=4)
    o.set_state(sinusoidal_ycyl(o))
    tke = [s.spectra()[3]["tke"]]
    for _ in range(20):
        assert s.step()["status"] == 0
        o.step()
        tke.append(s.spectra()[3]["tke"])
    check_criteria(tke, s.spectra_scales()[3])
    assert rel(s.get_state(gpu_mod.FIELD_UN), o.get_state()[1]) < (2e-5 if prec == 0 else 1e-11)
    o.close()
    s.close()


def test_rk4_refusals(gpu_mod):
    P = gpu_mod
    with pytest.raises(P.PsdnsError, match="velocity only"):
        P.Solver(n=32, precision=P.PREC_FP64, viscos=0.01, cfl=-1, dt=0.004, nc=1, pr=1.0, rkmethod=4)
    with pytest.raises(P.PsdnsError, match="rkmethod"):
        P.Solver(n=32, precision=P.PREC_FP64, viscos=0.01, cfl=-1, dt=0.004, rkmethod=3)
