"""Learned coarse solver (spectral-correction network): the device's
forward, backward and loss kernels against the FP64 restatement in
oracle/mlp.py (which is itself pinned by central finite differences), the
training kernel, the spectral filter and shell damping, and the protocol at
256^3 -> 64^3 (the bench runs 512^3 -> 128^3): the trained network must
bring the coarse box's E(k) and dissipation closer to the filtered fine DNS
than the plain coarse solver does.

Tolerances: gradients (BF16 weights on both sides, FP32 accumulation on the
device) 2e-3 relative to the largest component, network outputs 1e-5
relative; filtered shell energies 1e-6."""
import numpy as np
import pytest

from oracle import mlp


def _batch(rng, nb):
    x = np.stack([rng.uniform(0.05, 1.0, nb), rng.uniform(-2, 2, nb), rng.uniform(-1, 0.5, nb)], 1)
    a = rng.uniform(0.01, 0.5, nb)
    tau = rng.uniform(-0.05, 0.3, nb)
    wt = (rng.random(nb) > 0.2).astype(np.float64)
    return x, a, tau, wt


def test_oracle_gradient_against_finite_differences():
    rng = np.random.default_rng(3)
    w = rng.standard_normal(mlp.NP) * 0.3
    x, a, tau, wt = _batch(rng, 50)
    _, g = mlp.loss_and_grad(w, x, a, tau, wt)
    idx = rng.choice(mlp.NP, 40, replace=False)
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mlp.loss_and_grad(wp, x, a, tau, wt)[0] - mlp.loss_and_grad(wm, x, a, tau, wt)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g).max()), (i, fd, g[i])


@pytest.mark.gpu
def test_device_forward_and_gradient_against_oracle(gpu_mod):
    P = gpu_mod
    rng = np.random.default_rng(5)
    net = P.Corrector(11)
    w = (rng.standard_normal(mlp.NP) * 0.3).astype(np.float32)
    net.set_params(w)
    np.testing.assert_array_equal(net.get_params(), w)
    wb = mlp.bf16_round(w)
    x, a, tau, wt = _batch(rng, 3000)
    g_dev = net.forward(x)
    g_ref, _ = mlp.forward(wb, x)
    assert np.max(np.abs(g_dev - g_ref) / np.maximum(np.abs(g_ref), 1e-3)) < 1e-5
    grad_dev, loss_dev = net.grad(x, a, tau, wt)
    loss_ref, grad_ref = mlp.loss_and_grad(wb, x.astype(np.float32), a.astype(np.float32),
                                          tau.astype(np.float32), wt)
    assert abs(loss_dev - loss_ref) <= 1e-5 * loss_ref
    err = np.abs(grad_dev - grad_ref).max() / np.abs(grad_ref).max()
    print(f"device gradient vs FP64 oracle: max abs error / max |grad| = {err:.2e}")
    assert err < 2e-3
    net.close()


@pytest.mark.gpu
def test_device_training_fits_a_known_viscosity(gpu_mod):
    """Targets from a known g*(x): Adam on the device drives the loss down."""
    P = gpu_mod
    rng = np.random.default_rng(9)
    x, a, _, _ = _batch(rng, 4000)
    gstar = 0.5 + 3.0 * x[:, 0] ** 2 * np.exp(0.3 * x[:, 1])
    tau = a * gstar
    wt = np.ones(len(x))
    net = P.Corrector(2)
    hist = net.train(x, a, tau, wt, iters=1500, lr=3e-3)
    print(f"training loss {hist[0]:.3e} -> {hist[-1]:.3e}")
    assert hist[-1] < 0.02 * hist[0]
    g = net.forward(x)
    assert np.sqrt(np.mean((g - gstar) ** 2)) < 0.1 * np.sqrt(np.mean(gstar ** 2))
    net.close()


@pytest.mark.gpu
def test_filter_and_shell_factor(gpu_mod):
    P = gpu_mod
    import learned
    nu = learned.fine_viscosity(128)
    fine = P.Solver(learned.c5_params(128, nu, 1e-3))
    fine.field_init(77)
    for _ in range(3):
        fine.step()
    coarse = P.Solver(learned.c5_params(64, nu, 1e-3))
    coarse.filter_from(fine)
    K = P.resolved_shells(64)
    ef = fine.spectra(P.FIELD_UN)[0]
    ec = coarse.spectra(P.FIELD_UN)[0]
    np.testing.assert_allclose(ec[1:K - 1], ef[1:K - 1], rtol=1e-6)
    np.testing.assert_array_equal(coarse.get_state(P.FIELD_U), coarse.get_state(P.FIELD_UN))
    f = np.ones(K + 1)
    f[1:] = np.linspace(1.0, 0.5, K)
    coarse.shell_factor(f)
    ec2 = coarse.spectra(P.FIELD_UN)[0]
    np.testing.assert_allclose(ec2[1:K - 1], ec[1:K - 1] * f[1:K - 1] ** 2, rtol=1e-5)
    fine.close()
    coarse.close()


@pytest.mark.gpu
def test_learned_coarse_solver_beats_the_plain_coarse_solver(gpu_mod):
    """256^3 forced DNS (kmax eta = 1.5) filtered to 64^3 (kmax eta = 0.37):
    after training on 60 five-step windows, 400 steps of the corrected and of
    the plain 64^3 box from the same filtered state, same forcing.  The
    corrected box must track the filtered DNS within 5% in E(k) (mean over
    shells 4 .. K-1 and records), resolved dissipation and du/dx skewness,
    and closer than the plain coarse box on each."""
    import learned
    rep, net = learned.run(n_fine=256, n_coarse=64, dt=1e-3, spin=600, pairs=60, m=5, iters=2000, steps=400,
                           every=20)
    print("learned 256^3 -> 64^3:", rep)
    assert rep["fallbacks"] == 0 and rep["fine_status_errors"] == 0
    assert rep["loss_last"] < 0.1 * rep["loss_first"]
    for key in ("ek_mean_rel", "eps_rel", "skewness_rel"):
        assert rep["corr"][key] < rep["plain"][key], key
        assert rep["corr"][key] < 0.05, key
    net.close()
