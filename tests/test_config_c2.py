"""The 256^3 configuration with every part of the path on: FP32 device state,
Eswaran-Pope forcing (kforce 2.99, tforce 0.5, epsilon 0.1), viscosity from
kmax eta = 1.5, adaptive dt at Courant number 0.5 (cfl = pi), one passive
scalar with mean gradient G = (0, 1, 0) and Sc = 1, and 2^16 particles; two
RK2 steps against the FP64 oracle.

Tolerances (FP32 FFTs, ~1e-7 per operation): relative L2 of the velocity and
of the scalar 2e-5; particle positions 1e-6 n; particle velocities 2e-4 of
the largest."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_forced_scalar_particles_256(oracle_mod, gpu_mod):
    n = 256
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
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP32, viscos=nu, cfl=cfl, dt=0.0, kshift=1, kforce=kforce,
                       tforce=tforce, epsfor=epsfor, tfiuo=0.0, nc=1, pr=1.0, grad=(0.0, 1.0, 0.0))
    s.set_state(un0)
    s.particles_set(pos)
    for _ in range(2):
        assert o.step() == 0
        info = s.step()
        assert info["status"] == 0
        so = o.scalars()
        assert abs(info["dt"] - so["dt"]) <= 1e-5 * so["dt"]
    _, un_o = o.get_state()
    un_g = s.get_state(gpu_mod.FIELD_UN)
    assert rel_l2(un_g[:3], un_o[:3]) < 2e-5
    assert np.abs(un_o[3]).max() > 0
    assert rel_l2(un_g[3], un_o[3]) < 2e-5
    po, vo = o.particles_get()
    pg, vg = s.particles_get()
    assert np.abs(pg - po).max() < 1e-6 * n
    assert np.abs(vg - vo).max() < 2e-4 * np.abs(vo).max()
    o.close()
    s.close()
