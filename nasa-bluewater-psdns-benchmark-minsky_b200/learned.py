"""Learned coarse solver: a coarse box (n_c^3) advanced by the plain RK2 step
plus the spectral-correction network (psdns_gpu_corrector_*), trained on
filtered fine-box (n_f^3) DNS that the library itself produces, and judged
against that filtered DNS on the reference's statistics: E(k) and epsilon
(PSDNS/homogeneous/sptr.f:354-365) and the du/dx skewness from the moments
of PSDNS/vgmomt.f.

Protocol (all boxes on one GPU, FP32 state, same viscosity, same fixed dt):
* the fine box starts from the seeded field.f field; the coarse boxes start
  from its filter (psdns_gpu_filter_state: the fine modes inside the coarse
  truncation sphere).  Every box takes every step, so their RNG streams (grid
  shifts, Eswaran-Pope forcing) stay identical: the forcing of the coarse
  boxes is the fine box's.
* spin-up: `spin` steps.
* training data: `pairs` windows of `m` steps.  At the start of a window the
  plain coarse box is reset to the filter of the fine box and its per-shell
  features x(i) are taken; after m steps its shell energies E_c(i) are set
  against those of the filtered fine box E_f(i).  Target: the log damping
  tau(i) = ln(E_c / E_f) that an eddy viscosity nu g(i) causes as
  a(i) g(i), a(i) = 2 nu i^2 m dt; shells 4 .. K-1 (forcing shells and the
  partial last shell excluded).
* training: full-batch Adam on the device (psdns_gpu_corrector_train).
* evaluation: from the filter of the fine box after training, `steps` steps
  of the plain coarse box and of the corrected one (psdns_gpu_corrector_apply
  after each step), statistics recorded every `every` steps against the
  filtered fine box.
"""
import math
import time

import numpy as np

import psdns_gpu as P


def c5_params(n, nu, dt, forced=True, dft=0):
    return P.default_params(n=n, precision=P.PREC_FP32, viscos=nu, cfl=-1.0, dt=dt, kshift=1,
                            kforce=2.99 if forced else 0.0, tforce=0.5,
                            epsfor=0.1 / (4.0 * (4.0 * math.pi / 3.0) * 27.0), tfiuo=0.0, dft=dft)


def fine_viscosity(n_fine, eps=0.1):
    """nu with kmax eta = 1.5 on the fine grid (kmax = sqrt(2) n / 3)."""
    kmax = math.sqrt(2.0) * n_fine / 3.0
    return (1.5 / kmax) ** (4.0 / 3.0) * eps ** (1.0 / 3.0)


def du_dx_skewness(s):
    m, _ = s.gradient_moments(P.FIELD_UN)
    return m[2] / m[1] ** 1.5


class Boxes:
    def __init__(self, n_fine=512, n_coarse=128, dt=1e-3, seed=1234, forced=True):
        self.nf, self.nc, self.dt = n_fine, n_coarse, dt
        self.nu = fine_viscosity(n_fine)
        self.fine = P.Solver(c5_params(n_fine, self.nu, dt, forced))
        self.fine.field_init(seed)
        self.plain = P.Solver(c5_params(n_coarse, self.nu, dt, forced))
        self.corr = P.Solver(c5_params(n_coarse, self.nu, dt, forced))
        self.probe = P.Solver(c5_params(n_coarse, self.nu, dt, forced))
        for b in (self.plain, self.corr, self.probe):
            b.filter_from(self.fine)
        self.K = P.resolved_shells(n_coarse)
        self.t_fine = 0.0
        self.t_coarse = 0.0
        self.n_fine_steps = 0
        self.fallbacks = 0
        self.max_courant = 0.0
        self.status_errors = 0

    def close(self):
        for b in (self.fine, self.plain, self.corr, self.probe):
            b.close()

    def step(self, net=None):
        """One step of every box (the corrected box gets the network's
        correction after its step when net is given)."""
        t0 = time.perf_counter()
        info = self.fine.step()
        self.fine.sync()
        t1 = time.perf_counter()
        self.plain.step()
        self.probe.step()
        t2 = time.perf_counter()
        self.corr.step()
        if net is not None:
            ok, _ = self.corr.corrector_apply(net)
            self.fallbacks += 0 if ok else 1
        self.corr.sync()
        t3 = time.perf_counter()
        self.t_fine += t1 - t0
        self.t_coarse += t3 - t2
        self.n_fine_steps += 1
        self.max_courant = max(self.max_courant, info["courant"])
        self.status_errors += info["status"] != 0

    def shell_energy(self, box):
        return box.spectra(P.FIELD_UN)[0][:self.K + 1]


def training_data(bx, pairs=80, m=5):
    """(x, a, tau, w) rows for every resolved shell of every window."""
    X, A, T, W = [], [], [], []
    i = np.arange(1, bx.K + 1, dtype=np.float64)
    for _ in range(pairs):
        bx.plain.filter_from(bx.fine)
        x = bx.plain.corrector_features(P.FIELD_UN, bx.K)
        for _ in range(m):
            bx.step()
        ec = bx.shell_energy(bx.plain)[1:]
        bx.probe.filter_from(bx.fine)
        ef = bx.shell_energy(bx.probe)[1:]
        ok = (ec > 0) & (ef > 0) & (i >= 4) & (i <= bx.K - 1)
        tau = np.where(ok, np.log(np.where(ok, ec, 1.0) / np.where(ok, ef, 1.0)), 0.0)
        X.append(x)
        A.append(2.0 * bx.nu * i ** 2 * m * bx.dt)
        T.append(tau)
        W.append(ok.astype(np.float64))
    return (np.concatenate(X).astype(np.float32), np.concatenate(A).astype(np.float32),
            np.concatenate(T).astype(np.float32), np.concatenate(W).astype(np.float32))


def evaluate(bx, net, steps=400, every=20):
    """Statistics of the plain and the corrected coarse boxes against the
    filtered fine box, from the filter of the fine box's current state."""
    bx.plain.filter_from(bx.fine)
    bx.corr.filter_from(bx.fine)
    bx.t_fine = bx.t_coarse = 0.0
    bx.fallbacks = 0
    rec = {"plain": [], "corr": [], "dns": []}
    for k in range(1, steps + 1):
        bx.step(net)
        if k % every == 0:
            bx.probe.filter_from(bx.fine)
            for name, box in (("dns", bx.probe), ("plain", bx.plain), ("corr", bx.corr)):
                ek, _, _, st = box.spectra(P.FIELD_UN)
                rec[name].append((ek[:bx.K + 1].copy(), st["eps"], du_dx_skewness(box)))
    i = np.arange(bx.K + 1)
    shells = (i >= 4) & (i <= bx.K - 1)
    out = {}
    for name in ("plain", "corr"):
        ek_err, eps_err, sk_err = [], [], []
        for (ec, epc, skc), (ef, epf, skf) in zip(rec[name], rec["dns"]):
            ek_err.append(np.abs(ec[shells] - ef[shells]) / ef[shells])
            eps_err.append(abs(epc - epf) / epf)
            sk_err.append(abs(skc - skf) / abs(skf))
        ek_err = np.array(ek_err)
        out[name] = {"ek_mean_rel": float(ek_err.mean()), "ek_max_rel": float(ek_err.max()),
                     "eps_rel": float(np.mean(eps_err)), "skewness_rel": float(np.mean(sk_err))}
    out["dns_last"] = {"eps_resolved": rec["dns"][-1][1], "du_dx_skewness": rec["dns"][-1][2]}
    out["fallbacks"] = bx.fallbacks
    out["fine_max_courant"] = bx.max_courant
    out["fine_status_errors"] = bx.status_errors
    out["ms_per_step_fine"] = 1e3 * bx.t_fine / steps
    out["ms_per_step_coarse_corrected"] = 1e3 * bx.t_coarse / steps
    return out


def run(n_fine=512, n_coarse=128, dt=1e-3, spin=600, pairs=80, m=5, iters=3000, lr=3e-3, steps=400, every=20,
        seed=1234, net_seed=7):
    """The whole protocol; returns (report dict, trained Corrector)."""
    t0 = time.perf_counter()
    bx = Boxes(n_fine, n_coarse, dt, seed)
    try:
        for _ in range(spin):
            bx.step()
        X, A, T, W = training_data(bx, pairs, m)
        t_data = time.perf_counter() - t0
        net = P.Corrector(net_seed)
        t1 = time.perf_counter()
        hist = net.train(X, A, T, W, iters=iters, lr=lr)
        t_train = time.perf_counter() - t1
        ev = evaluate(bx, net, steps, every)
    finally:
        bx.close()
    ev.update({"n_fine": n_fine, "n_coarse": n_coarse, "dt": dt, "viscosity": bx.nu, "spin_up_steps": spin,
               "training_windows": pairs, "window_steps": m, "samples": int(len(X)), "adam_iters": iters,
               "loss_first": float(hist[0]), "loss_last": float(hist[-1]), "data_s": t_data, "train_s": t_train})
    return ev, net
