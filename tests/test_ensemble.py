"""Ensembles: boxes of uneven n, viscosity, dt mode and seed advanced together
with batched kernels (and CUDA graphs for fixed dt).  Each box must equal,
bit for bit, a single-box run of the same parameters; single-box runs are
checked against the oracle by the parity tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOXES = [  # (n, viscosity, cfl, dt, kshift, seed_input, field seed)
    (32, 0.01, -1.0, 0.004, 1, 122929298, 11),
    (48, 0.02, -1.0, 0.003, 1, 5551, 12),
    (32, 0.005, -1.0, 0.002, 2, 777, 13),
    (64, 0.01, 1.0, 0.0, 1, 122929298, 14),
    (32, 0.03, 1.5, 0.0, 3, 4242, 15),
    (48, 0.01, -1.0, 0.004, 4, 99, 16),
]


def _params(gpu_mod, prec, b):
    n, nu, cfl, dt, ks, seed, _ = b
    return gpu_mod.default_params(n=n, precision=prec, viscos=nu, cfl=cfl, dt=dt, kshift=ks, seed_input=seed)


@pytest.mark.parametrize("prec", [0, 1])
def test_ensemble_boxes_equal_single_runs(gpu_mod, prec):
    steps = 3
    ens = gpu_mod.Ensemble([_params(gpu_mod, prec, b) for b in BOXES])
    ens.field_init([b[6] for b in BOXES])
    rc, info = ens.step(steps)
    assert rc == 0
    for i, b in enumerate(BOXES):
        s = gpu_mod.Solver(_params(gpu_mod, prec, b))
        s.field_init(b[6])
        for _ in range(steps):
            si = s.step()
        np.testing.assert_array_equal(ens.get_state(i, gpu_mod.FIELD_UN), s.get_state(gpu_mod.FIELD_UN))
        np.testing.assert_array_equal(ens.get_state(i, gpu_mod.FIELD_U), s.get_state(gpu_mod.FIELD_U))
        assert info[i, 0] == si["dt"] and info[i, 1] == si["time"] and info[i, 7] == steps
        np.testing.assert_array_equal(info[i, 4:7], si["gsh1"])
        assert info[i, 2] == si["velmax"]
        # shell sums use atomics: equal to summation order
        e1 = ens.spectra(i)[3]["tke"]
        e2 = s.spectra()[3]["tke"]
        assert abs(e1 - e2) <= 1e-12 * abs(e2)
        s.close()
    ens.close()


def test_ensemble_set_state_round_trip_and_graph_replay(gpu_mod, oracle_mod):
    """set_state per box, then many fixed-dt steps (graph replays) against
    the oracle."""
    n, nu, dt = 32, 0.01, 0.004
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=dt, kshift=1)
    un0 = o.field_init(321)
    o.set_state(un0)
    p = gpu_mod.default_params(n=n, precision=1, viscos=nu, cfl=-1.0, dt=dt, kshift=1)
    ens = gpu_mod.Ensemble([p, p])
    ens.set_state(0, un0)
    ens.set_state(1, un0 * 0.5)
    np.testing.assert_array_equal(ens.get_state(0), un0)
    for _ in range(6):
        assert o.step() == 0
    rc, info = ens.step(6)
    assert rc == 0
    _, un_o = o.get_state()
    g = ens.get_state(0)
    assert np.linalg.norm(g - un_o) / np.linalg.norm(un_o) < 1e-11
    assert np.abs(ens.get_state(1)).max() > 0
    ens.close()
    o.close()


def test_ensemble_rejects_mixed_precision(gpu_mod):
    a = gpu_mod.default_params(n=32, precision=0, cfl=-1.0, dt=0.01)
    b = gpu_mod.default_params(n=32, precision=1, cfl=-1.0, dt=0.01)
    with pytest.raises(gpu_mod.PsdnsError):
        gpu_mod.Ensemble([a, b])


@pytest.mark.parametrize("prec", [0, 1])
def test_tile_autotuner_keeps_results_bit_identical(gpu_mod, prec):
    """Fixed-dt classes through the whole tuning (boxes per launch, then the
    K2 and K4 tiles, two steps per candidate) and on into the captured graph:
    every class reports a tuned choice, and every box equals its single-box
    run to roundoff (a tile variant is another compiled instance of the
    kernel, whose floating-point contraction may differ: FP64 1e-14, FP32
    1e-6 relative L2; the sub-batch size alone changes nothing, see above)."""
    boxes = [b for b in BOXES if b[2] < 0] + [(64, 0.02, -1.0, 0.003, 1, 31, 21), (64, 0.01, -1.0, 0.004, 3, 32, 22)]
    steps = 36
    ens = gpu_mod.Ensemble([_params(gpu_mod, prec, b) for b in boxes])
    ens.field_init([b[6] for b in boxes])
    rc, info = ens.step(steps)
    assert rc == 0
    tun = ens.tuning()
    assert len(tun) == 3 and all(t["tuned"] == 1 for t in tun), tun
    print("tuner:", tun)
    for i, b in enumerate(boxes):
        s = gpu_mod.Solver(_params(gpu_mod, prec, b))
        s.field_init(b[6])
        for _ in range(steps):
            s.step()
        a, b_ = ens.get_state(i, gpu_mod.FIELD_UN), s.get_state(gpu_mod.FIELD_UN)
        assert np.linalg.norm(a - b_) / np.linalg.norm(b_) < (1e-14 if prec else 1e-6)
        s.close()
    ens.close()
