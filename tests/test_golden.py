"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py with the
oracle): the oracle must reproduce them bit-for-bit on CPU, and the GPU path
must match them within the FP64 tolerance.  The reference itself ships no
golden vectors, so these pin regressions, not the reference."""
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load():
    return np.load(os.path.join(HERE, "rk2_forced_16.npz"))


def _oracle_run(oracle_mod, g):
    n = int(g["n"])
    o = oracle_mod.Oracle(n, float(g["viscos"]), cfl=-1.0, dt=float(g["dt"]), kshift=1,
                          seed_input=int(g["seed_input"]))
    o.set_forcing(float(g["kforce"]), float(g["tforce"]), float(g["epsfor"]), 0.0)
    return o


def test_oracle_reproduces_golden(oracle_mod):
    oracle_mod.set_threads(1)
    g = _load()
    o = _oracle_run(oracle_mod, g)
    un0 = o.field_init(int(g["seed_field"]))
    np.testing.assert_array_equal(un0, g["un0"])
    o.set_state(un0)
    o.particles_set(g["pos0"])
    for k in range(3):
        o.step()
        np.testing.assert_array_equal(o.scalars()["gsh"], g["gsh"][k])
    u, un = o.get_state()
    np.testing.assert_array_equal(un, g["un"])
    np.testing.assert_array_equal(u, g["u"])
    tab, efkz = o.forcing()
    np.testing.assert_array_equal(tab, g["forcing"])
    pos, vel = o.particles_get()
    np.testing.assert_array_equal(pos, g["pos"])
    np.testing.assert_array_equal(o.rann2(5, 32), g["rann2"])
    o.close()


def test_geometry_golden(oracle_mod):
    geo = np.load(os.path.join(HERE, "geometry.npz"))
    for m in (16, 64, 256, 1024):
        o = oracle_mod.Oracle(m, 0.01, kshift=4)
        assert o.xz_tot == int(geo[f"xz_tot_{m}"])
        np.testing.assert_array_equal(o.geometry()["cut"], geo[f"cut_{m}"])
        o.close()


@pytest.mark.gpu
def test_gpu_matches_golden(gpu_mod):
    g = _load()
    n = int(g["n"])
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=float(g["viscos"]), cfl=-1.0, dt=float(g["dt"]),
                       kshift=1, seed_input=int(g["seed_input"]), kforce=float(g["kforce"]),
                       tforce=float(g["tforce"]), epsfor=float(g["epsfor"]), tfiuo=0.0)
    s.field_init(int(g["seed_field"]))
    un0 = s.get_state(gpu_mod.FIELD_UN)
    assert np.linalg.norm(un0 - g["un0"]) / np.linalg.norm(g["un0"]) < 1e-13
    s.set_state(g["un0"])
    s.particles_set(g["pos0"])
    for k in range(3):
        info = s.step()
        np.testing.assert_array_equal(info["gsh1"], g["gsh"][k][:, 0])
    un = s.get_state(gpu_mod.FIELD_UN)
    assert np.linalg.norm(un - g["un"]) / np.linalg.norm(g["un"]) < 1e-11
    np.testing.assert_array_equal(s.forcing_table(), g["forcing"])
    pos, vel = s.particles_get()
    assert np.abs(pos - g["pos"]).max() < 1e-10 * n
    ek, dk, _, st = s.spectra()
    m = g["ek"] > 1e-12
    np.testing.assert_allclose(ek[m], g["ek"][m], rtol=1e-10)
    s.close()
