"""Passive scalar (nc = 1): advection by the velocity and by a uniform mean
gradient, diffusion with the Schmidt-number integrating factors
(PSDNS/step.f:387-407, homogeneous/proc4a.f:507-522, proc4b.f:69-75).

CPU: the oracle against closed forms of the RK2 recurrence.
GPU: the sm_100a path against the oracle through the C-ABI, with the
tolerances of the velocity parity tests (relative L2 of the scalar state:
FP64 1e-11, FP32 2e-5)."""
import numpy as np
import pytest


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_scalar_without_velocity_only_diffuses(oracle_mod):
    """u = 0: the advection term vanishes, so each step multiplies every
    scalar mode by xdif ydif zdif = exp(-nu k^2 dt / Sc), and the mean is
    zeroed (proc4b.f:200-205)."""
    n, nu, dt, sc = 16, 0.05, 0.01, 0.7
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=dt, kshift=1)
    o.set_scalar(pr=sc, grad=(0.3, -1.0, 0.5))
    rng = np.random.default_rng(5)
    un = np.zeros(o.state_shape(), complex)
    un[3] = rng.standard_normal(un[3].shape) + 1j * rng.standard_normal(un[3].shape)
    geo = o.geometry()
    # zero the points outside the sphere, which every stage zeroes as well
    ky = np.where(np.arange(n) > n // 2, np.arange(n) - n, np.arange(n))
    kz = np.where(geo["az"] > n // 2, geo["az"] - n, geo["az"])
    kx = np.repeat(np.arange(len(geo["colstart"]) - 1), np.diff(geo["colstart"]))
    k2 = kx[:, None] ** 2 + ky[None, :] ** 2 + kz[:, None] ** 2
    inside = (np.abs(ky)[None, :] <= geo["kymax"][:, None]) & (np.arange(n) != n // 2)[None, :]
    un[3][~inside] = 0
    o.set_state(un)
    steps = 3
    for _ in range(steps):
        assert o.step() == 0
    _, out = o.get_state()
    expect = un[3] * np.exp(-nu * k2 * dt / sc) ** steps
    expect[0, 0] = 0
    np.testing.assert_allclose(out[3], expect, rtol=1e-13, atol=1e-14)
    assert np.abs(out[:3]).max() == 0
    o.close()


def test_mean_gradient_source_on_a_shear_mode(oracle_mod):
    """u = (sin y, 0, 0) and grad = (G, 0, 0): the advection term is
    G sin(y) exp(-nu t); theta = a(t) sin y follows the integrating-factor
    Heun recurrence a' = f_s (a - dt/2 G e_n) - dt/2 G e_{n+1}, with
    e_n = exp(-nu t_n) and f_s = exp(-nu dt / Sc)."""
    n, nu, dt, sc, G = 16, 0.05, 0.01, 0.7, 0.3
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=dt, kshift=1)
    o.set_scalar(pr=sc, grad=(G, 0.0, 0.0))
    un = np.zeros(o.state_shape(), complex)
    un[0, 0, 1] = -0.5j
    un[0, 0, n - 1] = 0.5j
    o.set_state(un)
    a = 0.0
    fs = np.exp(-nu * dt / sc)
    for s in range(4):
        assert o.step() == 0
        e0, e1 = np.exp(-nu * s * dt), np.exp(-nu * (s + 1) * dt)
        a = fs * (a - 0.5 * dt * G * e0) - 0.5 * dt * G * e1
    _, out = o.get_state()
    np.testing.assert_allclose(out[3, 0, 1], -0.5j * a, rtol=1e-12)
    np.testing.assert_allclose(out[3, 0, n - 1], 0.5j * a, rtol=1e-12)
    out[3, 0, 1] = out[3, 0, n - 1] = 0
    assert np.abs(out[3]).max() < 1e-15


def test_scalar_is_passive_in_the_oracle(oracle_mod):
    """The velocity of a run with a scalar equals, bit for bit, the velocity
    of the same run without one."""
    n, nu = 16, 0.01
    runs = []
    for with_scalar in (False, True):
        o = oracle_mod.Oracle(n, nu, cfl=1.0, dt=0.005, kshift=1)
        if with_scalar:
            o.set_scalar(pr=0.5, grad=(0.0, 1.0, 0.0))
        un = o.field_init(4321)
        o.set_state(un)
        for _ in range(2):
            assert o.step() == 0
        runs.append(o.get_state()[1][:3].copy())
        o.close()
    np.testing.assert_array_equal(runs[0], runs[1])


def _scalar_pair(oracle_mod, gpu_mod, n, prec, steps, cfl, theta_seed, pr=0.7, grad=(0.2, 1.0, -0.3),
                 nu=0.01, dt=0.005):
    o = oracle_mod.Oracle(n, nu, cfl=cfl, dt=dt, kshift=1)
    o.set_scalar(pr=pr, grad=grad)
    un0 = o.field_init(1234)
    if theta_seed:
        # a random real scalar field: one component of another solenoidal field
        un0[3] = o.field_init(theta_seed)[0]
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=cfl, dt=dt, kshift=1, nc=1, pr=pr, grad=grad)
    s.set_state(un0)
    for _ in range(steps):
        assert o.step() == 0
        assert s.step()["status"] == 0
    u_o, un_o = o.get_state()
    out = (u_o, un_o, s.get_state(gpu_mod.FIELD_U), s.get_state(gpu_mod.FIELD_UN))
    o.close()
    s.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("n,steps,cfl,theta_seed", [(16, 2, -1.0, 77), (32, 3, 1.0, 77), (64, 2, 1.0, 0)])
def test_fp64_scalar_steps_match_oracle(oracle_mod, gpu_mod, n, steps, cfl, theta_seed):
    u_o, un_o, u_g, un_g = _scalar_pair(oracle_mod, gpu_mod, n, gpu_mod.PREC_FP64, steps, cfl, theta_seed)
    assert np.abs(un_o[3]).max() > 0
    assert rel_l2(un_g[3], un_o[3]) < 1e-11
    assert rel_l2(u_g[3], u_o[3]) < 1e-11
    assert rel_l2(un_g[:3], un_o[:3]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("n", [32, 64])
def test_fp32_scalar_steps_match_oracle(oracle_mod, gpu_mod, n):
    u_o, un_o, u_g, un_g = _scalar_pair(oracle_mod, gpu_mod, n, gpu_mod.PREC_FP32, 5, 1.0, 77)
    assert rel_l2(un_g[3], un_o[3]) < 2e-5
    assert rel_l2(u_g[3], u_o[3]) < 2e-5
    assert rel_l2(un_g[:3], un_o[:3]) < 2e-5


@pytest.mark.gpu
def test_gpu_velocity_is_unchanged_by_the_scalar(gpu_mod, oracle_mod):
    n, nu = 32, 0.01
    outs = []
    for nc in (0, 1):
        s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=nu, cfl=1.0, dt=0.005, kshift=1, nc=nc,
                           pr=0.7, grad=(0.0, 1.0, 0.0))
        o = oracle_mod.Oracle(n, nu)
        un0 = np.zeros(s.state_shape(), complex)
        un0[:3] = o.field_init(99)[:3]
        o.close()
        s.set_state(un0)
        for _ in range(2):
            assert s.step()["status"] == 0
        outs.append(s.get_state(gpu_mod.FIELD_UN)[:3].copy())
        s.close()
    assert rel_l2(outs[1], outs[0]) < 1e-14
