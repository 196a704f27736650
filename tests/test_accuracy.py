"""Accuracy of the device step against the FP64 oracle at the sizes the oracle
can run, closing the chain oracle -> FP64 device (256^3) on which the 1024^3
accuracy figures of bench.py rest (the FP64 device run is the judge there).

* FP64 device vs oracle at 256^3 with forcing, a passive scalar and 2^16
  particles (every part of the path on), two steps: state 1e-11 relative L2,
  particle positions 1e-11 n, particle velocities 1e-9 of the largest.
* Config C1 as stated: 64^3, FP64, nu = 0.01, dt = 0.005 (fixed), kshift 1,
  unforced, 20 steps from the seeded E(k) ~ k^4 exp(-2 (k/3)^2) field:
  E(k) per shell (sptr.f:161-165 shell index) 1e-10 relative and the final
  velocity 1e-11 relative L2.
* Config C2 over a longer horizon: 256^3 FP32 with forcing, scalar and 2^16
  particles, 20 steps against the FP64 oracle; the relative L2 error of the
  velocity is printed every step (error growth) and must stay below 1e-4,
  E(k) within 1e-4 in shells holding 1e-6 of the peak.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def c2_setup(oracle_mod, gpu_mod, n, prec):
    kmax = math.sqrt(2.0) * n / 3.0
    nu = (1.5 / kmax) ** (4.0 / 3.0) * 0.1 ** (1.0 / 3.0)
    kforce, tforce = 2.99, 0.5
    epsfor = 0.1 / (4.0 * (4.0 * math.pi / 3.0) * 3.0 ** 3)
    cfl = math.pi
    o = oracle_mod.Oracle(n, nu, cfl=cfl, dt=0.0, kshift=1)
    o.set_forcing(kforce, tforce, epsfor, 0.0)
    o.set_scalar(pr=1.0, grad=(0.0, 1.0, 0.0))
    un0 = o.field_init(1234)
    o.set_state(un0)
    rng = np.random.default_rng(1235)
    pos = 1.0 + rng.random((1 << 16, 3)) * n
    o.particles_set(pos)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=cfl, dt=0.0, kshift=1, kforce=kforce,
                       tforce=tforce, epsfor=epsfor, tfiuo=0.0, nc=1, pr=1.0, grad=(0.0, 1.0, 0.0))
    s.set_state(un0)
    s.particles_set(pos)
    return o, s


def test_fp64_256_every_part_on(oracle_mod, gpu_mod):
    n = 256
    o, s = c2_setup(oracle_mod, gpu_mod, n, gpu_mod.PREC_FP64)
    for _ in range(2):
        assert o.step() == 0
        info = s.step()
        assert info["status"] == 0
        so = o.scalars()
        assert abs(info["dt"] - so["dt"]) <= 1e-12 * so["dt"]
        assert abs(info["velmax"] - so["velmax"]) <= 1e-12 * so["velmax"]
    u_o, un_o = o.get_state()
    un_g = s.get_state(gpu_mod.FIELD_UN)
    u_g = s.get_state(gpu_mod.FIELD_U)
    assert rel_l2(un_g[:3], un_o[:3]) < 1e-11
    assert rel_l2(u_g[:3], u_o[:3]) < 1e-11
    assert rel_l2(un_g[3], un_o[3]) < 1e-11
    po, vo = o.particles_get()
    pg, vg = s.particles_get()
    assert np.abs(pg - po).max() < 1e-11 * n
    assert np.abs(vg - vo).max() < 1e-9 * np.abs(vo).max()
    o.close()
    s.close()


def test_config_c1_as_stated(oracle_mod, gpu_mod):
    n, nu, dt = 64, 0.01, 0.005
    o = oracle_mod.Oracle(n, nu, cfl=-1.0, dt=dt, kshift=1)
    un0 = o.field_init(1234)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=nu, cfl=-1.0, dt=dt, kshift=1)
    s.set_state(un0)
    errs = []
    for _ in range(20):
        assert o.step() == 0
        assert s.step()["status"] == 0
        errs.append(rel_l2(s.get_state(gpu_mod.FIELD_UN), o.get_state()[1]))
    print("C1 FP64 device vs oracle, relative L2 per step:", " ".join(f"{e:.2e}" for e in errs))
    _, un_o = o.get_state()
    un_g = s.get_state(gpu_mod.FIELD_UN)
    assert rel_l2(un_g, un_o) < 1e-11
    ek_o = o.spectra(1)[0]
    ek_g = s.spectra(gpu_mod.FIELD_UN)[0]
    m = ek_o > 0
    assert m.sum() >= 28   # shells 1 .. int(kmax + 1.5) hold energy (kmax = 30.2)
    assert np.max(np.abs(ek_g[m] - ek_o[m]) / ek_o[m]) < 1e-10
    o.close()
    s.close()


def test_config_c2_twenty_steps_error_growth(oracle_mod, gpu_mod):
    n = 256
    o, s = c2_setup(oracle_mod, gpu_mod, n, gpu_mod.PREC_FP32)
    errs = []
    for _ in range(20):
        assert o.step() == 0
        assert s.step()["status"] == 0
        _, un_o = o.get_state()
        errs.append(rel_l2(s.get_state(gpu_mod.FIELD_UN)[:3], un_o[:3]))
    print("C2 FP32 device vs FP64 oracle, velocity relative L2 per step:", " ".join(f"{e:.2e}" for e in errs))
    assert max(errs) < 1e-4, errs
    ek_o = o.spectra(1)[0]
    ek_g = s.spectra(gpu_mod.FIELD_UN)[0]
    m = ek_o > 1e-6 * ek_o.max()
    ek_err = np.max(np.abs(ek_g[m] - ek_o[m]) / ek_o[m])
    print(f"C2 after 20 steps: max relative E(k) error {ek_err:.2e} over {int(m.sum())} shells")
    assert ek_err < 1e-4
    po, _ = o.particles_get()
    pg, _ = s.particles_get()
    print(f"C2 after 20 steps: max particle position error {np.abs(pg - po).max():.2e} grid units")
    assert np.abs(pg - po).max() < 1e-4 * n
    o.close()
    s.close()
