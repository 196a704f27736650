#!/usr/bin/env python
"""bench.py -- throughput of the PSDNS RK2 time step on B200.

Workload: the forced 1024^3 box with an FP32 device state, advanced by the
RK2 step of PSDNS (both stages: phase shift, inverse transforms, products,
forward transforms, wavespace closure, integrating factor update, projection),
with Eswaran-Pope forcing on shells |k| < 3 (tforce = 0.5, epsilon target
0.1), viscosity from kmax*eta = 1.5, adaptive dt at Courant number 0.5
(cfl = pi) and 2^24 Lagrangian particles (FP64 positions, FP32 spline
coefficients).  The initial field is the seeded random solenoidal field of
field.f with E(k) ~ k^4 exp(-2 (k/3)^2), u' = 1, and particles start
uniformly at random (seeded); all data is synthetic.

`value` is points per second (Gpts/s = n^3 / step time) with the state
resident in HBM; `e2e` is the same metric through the C-ABI with the state in
pinned host memory, copied in and out every step (psdns_gpu_set_state_async /
psdns_gpu_get_state_async: chunked copies on their own streams, so that the
upload of a step overlaps the download of the one before).

Multi-GPU: one independent box per GPU (replicas only; the single-box path
has no data-path collective), timed as the max over ranks.

`--impl reference` times the CPU restatement of the reference's step (the
oracle, C/OpenMP on all host cores) on a bounded sample: one RK2 step of a
256^3 box per timed step.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "nasa-bluewater-psdns-benchmark-minsky_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

METRIC = "RK2 step throughput at 1024^3 (Gpts/s = N^3 / step time)"
UNIT = "Gpts/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--prec", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-n", type=int, default=256)
    ap.add_argument("--particles", type=int, default=1 << 24)
    ap.add_argument("--unforced", action="store_true")
    ap.add_argument("--nc", type=int, default=0, choices=[0, 1],
                    help="1: also advance a passive scalar (Sc = 1, mean gradient (0, 1, 0))")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision arm (1-D transforms on the tensor cores, split BF16)")
    ap.add_argument("--no-extra-arms", action="store_true",
                    help="skip the FP64-state and passive-scalar timings at 1024^3")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned arm (128^3 + spectral-correction network against 512^3 DNS)")
    ap.add_argument("--accuracy-steps", type=int, default=3,
                    help="steps of the same-seed FP64 run that judges the error of the timed arm (0: skip)")
    ap.add_argument("--dft-lines", type=int, default=0,
                    help="instead: the 1024-point line DFT on its own (FP32 Stockham and split-BF16 tensor cores), "
                         "L lines through psdns_gpu_dft_lines")
    ap.add_argument("--diagnostics", action="store_true",
                    help="time the diagnostics (shell spectra, 1-D spectra and scales, gradient "
                         "moments, transfer spectrum) on the --n box instead of the step")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="instead: B boxes of n in {32,48,64,96}, log-uniform viscosity, fixed dt")
    return ap.parse_args()


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_oracle_rate(n, steps, warmup, threads):
    """Oracle (FP64 C/OpenMP restatement of the reference step) on host cores."""
    from oracle import oracle
    oracle.build()
    oracle.set_threads(threads)
    o = oracle.Oracle(n, 0.01, cfl=-1.0, dt=0.001, kshift=1)
    o.set_state(o.field_init(1234))
    for _ in range(warmup):
        o.step()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        o.step()
        ts.append(time.perf_counter() - t0)
    o.close()
    return ts


def algorithmic_bytes(n, kxn, xz_tot, csz):
    """Compulsory HBM bytes per launch of the five stage kernels (per-axis pass
    model: each pass reads and writes its variables once, cylinder zero bands
    are neither read nor written, the x chain keeps the physical field on chip).
    C = xz_tot*n complex, Z = kxn*n^2 complex."""
    C = xz_tot * n * csz
    Z = kxn * n * n * csz
    return {"k_yinv": 6 * C, "k_zinv": 3 * C + 3 * Z, "k_xchain": 8 * Z, "k_zfwd": 5 * Z + 4 * C,
            "k_yfwd": 13 * C}, 2 * (26 * C + 16 * Z)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.dev), "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        sm, mx, reasons, n = [], [], set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            n += 1
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": n}


def reduce_max_ms(ms, dist, device):
    """Max over ranks of a per-rank time (the slowest replica sets the pace);
    device is "cuda" under NCCL, "cpu" under gloo."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, n, ms_step):
    """Whole-job Gpts/s: every replica advances its own n^3 box per step."""
    return world * n ** 3 / (ms_step * 1e-3) / 1e9


def accuracy_leg(P, n, make_solver, npart, steps, arms):
    """Error of each arm against the FP64 device run of the same seed and
    configuration after `steps` steps (run one after the other, outside the
    timed region; the FP64 device step matches the FP64 oracle to 1e-11 up
    to 256^3).  Returns, per arm: relative L2 of the velocity un, the largest
    relative E(k) error over shells holding at least 1e-6 of the peak (and,
    as the tail figure, 1e-10 of the peak; sptr.f:161-165 shells, FP64 sums
    on the device), and the largest
    particle position difference in grid units."""
    import numpy as np

    def run(prec, mode):
        s = make_solver(prec, mode)
        for _ in range(steps):
            s.step()
        out = {"un": s.get_state(P.FIELD_UN), "ek": s.spectra(P.FIELD_UN)[0]}
        if npart > 0:
            out["pos"] = s.particles_get()[0]
        s.close()
        return out

    ref = run(P.PREC_FP64, 0)
    nrm = np.sqrt(sum(float(np.vdot(ref["un"][v], ref["un"][v]).real) for v in range(ref["un"].shape[0])))
    res = {}
    for name, prec, mode in arms:
        got = run(prec, mode)
        d2 = 0.0
        for v in range(3):
            d = got["un"][v] - ref["un"][v]
            d2 += float(np.vdot(d, d).real)
            del d
        m = ref["ek"] > 1e-6 * ref["ek"].max()
        t = ref["ek"] > 1e-10 * ref["ek"].max()
        ent = {"velocity_rel_l2": math.sqrt(d2) / nrm,
               "ek_max_rel": float(np.max(np.abs(got["ek"][m] - ref["ek"][m]) / ref["ek"][m])),
               "ek_shells": int(m.sum()),
               "ek_max_rel_tail": float(np.max(np.abs(got["ek"][t] - ref["ek"][t]) / ref["ek"][t])),
               "ek_shells_tail": int(t.sum())}
        if npart > 0:
            ent["particle_pos_max"] = float(np.abs(got["pos"] - ref["pos"]).max())
        res[name] = ent
        del got
    return {"against": f"FP64 device run of the same seed and configuration, {steps} steps", "steps": steps,
            "arms": res}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = host_cores()
    n = args.cpu_n
    ts = cpu_oracle_rate(n, args.steps, args.warmup, cores)
    t = sum(ts) / len(ts)
    v = n ** 3 / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"RK2 step, {args.n}^3 box (timed on a bounded sample: one {n}^3 step per timed step)",
                   "n": args.n, "sample_n": n},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"one full RK2 step of a {n}^3 box per timed step (FP64 C/OpenMP restatement "
                                   f"of the reference, {cores} threads); Gpts/s = {n}^3/t"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ensemble(args):
    """Ensemble workload: B independent boxes, n uniform in {32, 48, 64, 96},
    viscosity log-uniform in [0.005, 0.05], seeds 1000 + i, the C1 spectrum
    and a fixed dt of 0.005 (cfl < 0), advanced together by batched kernels
    replayed from CUDA graphs.  Timed with the host clock around whole
    synchronised steps (the classes run on several streams); the same boxes
    advanced one context after the other give the unbatched comparison."""
    import numpy as np
    import torch
    import psdns_gpu as P
    torch.cuda.set_device(0)
    prec = P.PREC_FP32 if args.prec == "fp32" else P.PREC_FP64
    rng = np.random.default_rng(2024)
    B = args.ensemble
    ns = rng.choice([32, 48, 64, 96], size=B)
    nus = np.exp(rng.uniform(np.log(0.005), np.log(0.05), size=B))
    params = [P.default_params(n=int(ns[i]), precision=prec, viscos=float(nus[i]), cfl=-1.0, dt=0.005, kshift=1,
                               seed_input=122929298 + i) for i in range(B)]
    ens = P.Ensemble(params)
    ens.field_init([1000 + i for i in range(B)])
    # the first steps of each class tune it (boxes per launch, then the K2 and
    # K4 tiles: two steps per candidate, about 2 log2(boxes per class) + 14
    # steps), then the graph is captured
    warm = max(args.warmup, 40)
    ens.step(warm)
    t0 = time.perf_counter()
    rc, info = ens.step(args.steps)
    t = (time.perf_counter() - t0) / args.steps
    pts = float(sum(int(n) ** 3 for n in ns))
    tuning = ens.tuning()
    # unbatched comparison: separate contexts, one step each, one after the other
    ctxs = [P.Solver(p) for p in params]
    for i, c in enumerate(ctxs):
        c.field_init(1000 + i)
        c.step()
    k = 2
    t0 = time.perf_counter()
    for _ in range(k):
        for c in ctxs:
            c.step()
    t_sep = (time.perf_counter() - t0) / k
    for c in ctxs:
        c.close()
    ens.close()
    out = {"metric": "ensemble RK2 step throughput (Gpts/s = sum of n^3 / step time)", "value": pts / t / 1e9,
           "unit": "Gpts/s", "n_gpus": 1, "steps": args.steps, "warmup": warm,
           "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32" if prec == P.PREC_FP32 else "f64",
           "data": "synthetic: seeded random solenoidal fields, E(k)~k^4 exp(-2(k/3)^2), u'=1",
           "config": {"workload": f"ensemble of {B} boxes, n in {{32,48,64,96}}, log-uniform viscosity "
                                  "[0.005, 0.05], dt 0.005, unforced",
                      "boxes": B, "n_counts": {str(v): int((ns == v).sum()) for v in (32, 48, 64, 96)},
                      "timing": "host clock around synchronised ensemble steps"},
           "status": rc, "tuning": tuning, "separate_contexts_ms_per_step": t_sep * 1e3,
           "batching_speedup": t_sep / t}
    print(json.dumps(out), flush=True)
    return 0


def run_dft_lines(args):
    """The DFT primitive alone: L random complex lines of 1024 points through
    psdns_gpu_dft_lines in both modes (host copies included in the call),
    errors against numpy's float64 FFT."""
    import numpy as np
    import psdns_gpu as P
    rng = np.random.default_rng(1)
    L = args.dft_lines
    x = (rng.standard_normal((L, 1024)) + 1j * rng.standard_normal((L, 1024))).astype(np.complex64)
    x = x.astype(np.complex128)
    ref = np.fft.fft(x, axis=-1)
    out = {"metric": "1024-point line DFT", "lines": L}
    for name, mode in (("fp32_stockham", P.DFT_FP32), ("tc_bf16x3", P.DFT_TC_BF16X3)):
        t0 = time.perf_counter()
        y = P.dft_lines(x, mode)
        out[name] = {"rel_l2": float(np.linalg.norm(y - ref) / np.linalg.norm(ref)),
                     "call_s": time.perf_counter() - t0}
    print(json.dumps(out), flush=True)
    return 0


def run_diagnostics(args):
    """The diagnostics of the library on the bench's box (no particles): each
    call timed on the host around the synchronous C-ABI call (device work plus
    the small result copies), median of --steps calls after --warmup."""
    import math
    import statistics
    import torch
    import psdns_gpu as P
    torch.cuda.set_device(0)
    n = args.n
    prec = P.PREC_FP32 if args.prec == "fp32" else P.PREC_FP64
    kmax = math.sqrt(2.0) * n / 3.0
    nu = (1.5 / kmax) ** (4.0 / 3.0) * 0.1 ** (1.0 / 3.0)
    s = P.Solver(n=n, precision=prec, viscos=nu, cfl=math.pi, dt=0.0, kshift=1, kforce=2.99, tforce=0.5,
                 epsfor=0.1 / (4.0 * (4.0 * math.pi / 3.0) * 27.0), tfiuo=0.0)
    s.field_init(1234)
    for _ in range(2):
        s.step()
    s.sync()
    calls = {
        "spectra": lambda: s.spectra(P.FIELD_UN),
        "spectra_scales": lambda: s.spectra_scales(P.FIELD_UN),
        "gradient_moments": lambda: s.gradient_moments(P.FIELD_UN, (0.1, 0.2, 0.3)),
        "transfer_spectrum": lambda: s.transfer_spectrum((0.1, 0.2, 0.3)),
        "step": lambda: (s.step(), s.sync()),
    }
    out = {"metric": "diagnostics at %d^3 (ms per call, median)" % n, "n": n, "precision": args.prec,
           "timing": "host clock around each synchronous call"}
    for name, f in calls.items():
        for _ in range(max(1, args.warmup)):
            f()
        ts = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            f()
            ts.append((time.perf_counter() - t0) * 1e3)
        out[name + "_ms"] = statistics.median(ts)
    s.close()
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.diagnostics:
        return run_diagnostics(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.dft_lines > 0:
        return run_dft_lines(args)
    if args.ensemble > 0:
        return run_ensemble(args)
    import torch
    import psdns_gpu as P

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    # the library uses the current device of the calling thread
    n = args.n
    prec = P.PREC_FP32 if args.prec == "fp32" else P.PREC_FP64
    csz = 8 if prec == P.PREC_FP32 else 16
    import math
    import numpy as np
    eps_target = 0.1
    kmax = math.sqrt(2.0) * n / 3.0
    nu = (1.5 / kmax) ** (4.0 / 3.0) * eps_target ** (1.0 / 3.0)   # kmax*eta = 1.5
    kforce = 0.0 if args.unforced else 2.99                          # shells |k| < 3
    epsfor = eps_target / (4.0 * (4.0 * math.pi / 3.0) * 3.0 ** 3)   # epfor_param.f: eps/(4 N_f)
    s = P.Solver(n=n, precision=prec, viscos=nu, cfl=math.pi, dt=0.0, kshift=1,
                 kforce=kforce, tforce=0.5, epsfor=epsfor, tfiuo=0.0, nc=args.nc, pr=1.0, grad=(0.0, 1.0, 0.0))
    s.field_init(1234 + rank)
    npart = args.particles
    if npart > 0:
        rng = np.random.default_rng(4321 + rank)
        s.particles_set(1.0 + rng.random((npart, 3)) * n)
    stream = torch.cuda.ExternalStream(s.stream())

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        s.step()
    barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.4)
    s.profile(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        info = s.step()
    e1.record(stream)
    e1.synchronize()
    ms_total = e0.elapsed_time(e1)
    kms, kcnt = s.kernel_times()
    s.profile(False)
    ck = clocks.stop()
    barrier()
    ms_total = reduce_max_ms(ms_total, dist, "cuda")
    ms_step = ms_total / args.steps
    value = aggregate_rate(world, n, ms_step)

    names = ["k_yinv", "k_zinv", "k_xchain", "k_zfwd", "k_yfwd", "particles"]
    per_launch, step_bytes = algorithmic_bytes(n, s.kxn, s.xz_tot, csz)
    if npart > 0:
        # particle phase: one extra 3-variable backward chain (9C + 6Z), the
        # spline coefficients written once (3 values per point), two stencil
        # gathers (min of the whole coefficient field and 64 points x 3 values
        # per particle) and FP64 positions/velocities read and written
        C = s.xz_tot * n * csz
        Z = s.kxn * n * n * csz
        rsz = csz // 2
        coef = 3 * n ** 3 * rsz
        per_launch["particles"] = 9 * C + 6 * Z + coef + 2 * min(coef, npart * 64 * 3 * rsz) + npart * 12 * 8
        step_bytes += per_launch["particles"]
    else:
        per_launch["particles"] = 0
    dom = max(range(5), key=lambda i: kms[i])   # dominant stage kernel
    avg_ms = kms[dom] / max(1, kcnt[dom])
    achieved = per_launch[names[dom]] / (avg_ms * 1e-3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak = 6650.0
        peak_src = "fallback"
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        key = f"{names[dom]}_{args.prec}_{n}"
        if key in tj:
            traffic = tj[key]
    kernel_table = {names[i]: {"ms_per_launch": kms[i] / max(1, kcnt[i]), "launches": int(kcnt[i]),
                               "share": kms[i] / max(1e-12, sum(kms)),
                               "algorithmic_bytes": per_launch[names[i]],
                               "achieved_gbs": per_launch[names[i]] / (kms[i] / max(1, kcnt[i]) * 1e-3) / 1e9}
                    for i in range(6) if kcnt[i] > 0}

    # end to end through the C-ABI: state (complex(8), reference layout) copied
    # from pinned host memory and back every step
    e2e = None
    if not args.no_e2e:
        nbytes = (3 + args.nc) * s.xz_tot * n * 16
        try:
            host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            ptr = host.data_ptr()
            s.get_state_ptr(ptr)
            barrier()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            # each step: upload the state from pinned memory, step, download
            # the new state to the same buffer; the asynchronous calls let an
            # upload overlap the previous download chunk by chunk.  Headline:
            # the sphere copies (the entries inside the truncation sphere,
            # which are all the step reads and writes); beside it the copies
            # of the whole reference-layout array.
            def timed(up, down):
                barrier()
                f0.record(stream)
                for _ in range(args.e2e_steps):
                    up(ptr)
                    s.step()
                    down(ptr)
                s.sync()
                f1.record(stream)
                f1.synchronize()
                return reduce_max_ms(f0.elapsed_time(f1) / args.e2e_steps, dist, "cuda")
            ems_full = timed(s.set_state_async_ptr, s.get_state_async_ptr)
            ems = timed(s.set_state_sphere_async_ptr, s.get_state_sphere_async_ptr)
            # entries per variable inside the truncation sphere (masks.f)
            sphere_bytes = int(P.sphere_mask(n).sum()) * (3 + args.nc) * 16
            e2e = {"value": aggregate_rate(world, n, ems), "unit": UNIT, "h2d_bytes_per_step": sphere_bytes,
                   "d2h_bytes_per_step": sphere_bytes, "ms_per_step": ems, "steps": args.e2e_steps,
                   "copies": "entries inside the truncation sphere, pinned host memory read and written by kernels",
                   "full_array": {"value": aggregate_rate(world, n, ems_full), "ms_per_step": ems_full,
                                  "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}}
            del host
        except Exception as ex:  # pinned allocation may exceed host memory
            e2e = {"value": None, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                   "error": str(ex)[:200]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = host_cores()
        ts = cpu_oracle_rate(args.cpu_n, 1, 0, cores)
        t = sum(ts) / len(ts)
        cpu = {"value": args.cpu_n ** 3 / t / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"one RK2 step of a {args.cpu_n}^3 box (FP64 C/OpenMP restatement of the reference, "
                         f"{cores} threads, {t:.2f} s); Gpts/s = {args.cpu_n}^3/t"}
    s.close()

    def make_solver(p_, mode, nc=None):
        t = P.Solver(n=n, precision=p_, viscos=nu, cfl=math.pi, dt=0.0, kshift=1, kforce=kforce, tforce=0.5,
                     epsfor=epsfor, tfiuo=0.0, nc=args.nc if nc is None else nc, pr=1.0, grad=(0.0, 1.0, 0.0),
                     dft=mode)
        t.field_init(1234 + rank)
        if npart > 0:
            t.particles_set(1.0 + np.random.default_rng(4321 + rank).random((npart, 3)) * n)
        return t

    # mixed-precision arm: the same workload with every 1-D transform of the
    # five stage kernels on the tensor cores (split BF16, FP32 accumulation);
    # the particle spline chain keeps its FP32 transforms
    mixed = None
    use_mixed = n == 1024 and prec == P.PREC_FP32 and not args.no_mixed
    if use_mixed:
        try:
            t = make_solver(P.PREC_FP32, P.DFT_TC_BF16X3)
            tstream = torch.cuda.ExternalStream(t.stream())
            for _ in range(args.warmup):
                t.step()
            barrier()
            t.profile(True)
            e0.record(tstream)
            for _ in range(args.steps):
                t.step()
            e1.record(tstream)
            e1.synchronize()
            mms = reduce_max_ms(e0.elapsed_time(e1), dist, "cuda") / args.steps
            mk, mc = t.kernel_times()
            t.profile(False)
            t.close()
            mixed = {"ms_per_step": mms, "value": aggregate_rate(world, n, mms), "unit": UNIT,
                     "dft": "tensor cores (tcgen05.mma), split BF16 hi+lo, 3 products, FP32 accumulation",
                     "kernels": {names[i]: {"ms_per_launch": mk[i] / max(1, mc[i]), "launches": int(mc[i]),
                                            "achieved_gbs": per_launch[names[i]] / (mk[i] / max(1, mc[i]) * 1e-3) / 1e9}
                                 for i in range(6) if mc[i] > 0},
                     "gpu_launches": int(sum(mc[:5]) + 4 * mc[5])}
        except Exception as ex:
            mixed = {"error": str(ex)[:300]}
    # the same workload with an FP64 state, and with one passive scalar (Sc 1,
    # mean gradient (0, 1, 0)), timed like the plain arm (CUDA events on the
    # solver's stream, --warmup then --steps steps); one GPU only
    def timed_arm(t):
        tstream = torch.cuda.ExternalStream(t.stream())
        for _ in range(args.warmup):
            t.step()
        torch.cuda.synchronize()
        e0.record(tstream)
        for _ in range(args.steps):
            t.step()
        e1.record(tstream)
        e1.synchronize()
        return e0.elapsed_time(e1) / args.steps

    other_arms = {}
    if rank == 0 and world == 1 and n == 1024 and prec == P.PREC_FP32 and args.nc == 0 and not args.no_extra_arms:
        for name, p_, nc_ in (("fp64_state", P.PREC_FP64, 0), ("scalar_nc1_fp32", P.PREC_FP32, 1)):
            try:
                t = make_solver(p_, P.DFT_FP32, nc_)
                ams = timed_arm(t)
                t.close()
                other_arms[name] = {"ms_per_step": ams, "value": aggregate_rate(world, n, ams), "unit": UNIT,
                                    "particles": npart, "nc": nc_}
            except Exception as ex:
                other_arms[name] = {"error": str(ex)[:300]}
    # learned arm: 512^3 forced DNS (kmax eta = 1.5) against a 128^3 box with
    # the spectral-correction network, trained on the device on filtered
    # 512^3 data made in the same run (learned.py); wall time per step of
    # each and the corrected box's error against the filtered DNS
    learned_arm = None
    if rank == 0 and world == 1 and n == 1024 and not args.no_learned:
        try:
            import learned
            rep, net = learned.run(n_fine=512, n_coarse=128, dt=5e-4, spin=1200, pairs=60, m=10, iters=2000,
                                   steps=800, every=40)
            net.close()
            learned_arm = dict(rep)
            learned_arm["ms_per_step_plain_512"] = rep["ms_per_step_fine"]
            learned_arm["speedup_wall_time"] = rep["ms_per_step_fine"] / rep["ms_per_step_coarse_corrected"]
            learned_arm["timing"] = "host clock around each synchronised step (corrected: step + correction)"
        except Exception as ex:
            learned_arm = {"error": str(ex)[:300]}
    accuracy = None
    if rank == 0 and world == 1 and args.accuracy_steps > 0 and prec == P.PREC_FP32:
        arms = [("fp32", P.PREC_FP32, P.DFT_FP32)]
        if use_mixed:
            arms.append(("mixed_bf16x3", P.PREC_FP32, P.DFT_TC_BF16X3))
        try:
            accuracy = accuracy_leg(P, n, make_solver, npart, args.accuracy_steps, arms)
        except Exception as ex:
            accuracy = {"error": str(ex)[:300]}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == P.PREC_FP32 else "f64",
            "data": "synthetic: seeded random solenoidal field, E(k)~k^4 exp(-2(k/3)^2), u'=1",
            "config": {"workload": f"{'unforced' if kforce == 0 else 'forced'} RK2 step of one {n}^3 periodic box "
                                   f"per GPU, {args.prec} state, kshift=1 phase shifts, cfl=pi (Courant 0.5), "
                                   f"{npart} particles" + (", one passive scalar (Sc 1, G (0,1,0))" if args.nc else ""),
                       "nc": args.nc, "n": n, "precision": args.prec, "viscosity": nu, "kforce": kforce, "tforce": 0.5,
                       "epsfor": epsfor, "particles": npart, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (state >= 9 GB per variable set), no flush needed"},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                         "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "step_achieved": step_bytes / (ms_step * 1e-3) / 1e9,
                         "step_frac": step_bytes / (ms_step * 1e-3) / 1e9 / peak},
            "kernels": kernel_table,
            "arms": dict({"plain_fp32": {"ms_per_step": ms_step, "value": value, "unit": UNIT},
                          "mixed_bf16x3": mixed, "learned_128_vs_512": learned_arm}, **other_arms),
            "accuracy": accuracy,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(sum(kcnt[:5]) + 4 * kcnt[5]),
            "clocks": ck,
            "last_step": {"dt": info["dt"], "velmax": info["velmax"], "courant": info["courant"]},
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
