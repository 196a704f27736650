"""psdns_gpu_rk_stage_noalloc: the RK stage for callers that cannot call
cudaMalloc (for instance a driver whose device arrays belong to another
runtime, or one with a fixed device-memory budget).  It runs on the caller's
own device arrays with its scratch in a static device array, and must give the
same result as the context-based psdns_gpu_rk_stage (FP64: 1e-12 relative L2;
FP32: 1e-6, the same kernels on the same inputs), and the oracle's when it is
the first thing a process runs on the GPU (FP64: 1e-11, the tolerance of the
other FP64 device-against-oracle tests).

Collected last on purpose (file name), so that a run stopping at the first
failure has already run every other test."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GSHS = [np.array([[0.1, 0.6], [0.3, 0.8], [0.45, 0.95]]), np.array([[0.7, 0.2], [0.05, 0.55], [0.9, 0.4]])]


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("n,prec,tol", [(16, 1, 1e-12), (32, 1, 1e-12), (64, 1, 1e-12), (32, 0, 1e-6),
                                        (64, 0, 1e-6)])
def test_noalloc_stage_matches_context_stage(gpu_mod, n, prec, tol):
    import torch
    P = gpu_mod
    nu, dt = 0.01, 0.004
    ref = P.Solver(n=n, precision=prec, viscos=nu, cfl=-1.0, dt=dt, kshift=4)
    ref.field_init(31 + n)
    cdt = np.complex128 if prec == P.PREC_FP64 else np.complex64
    u0 = ref.get_state(P.FIELD_U).astype(cdt)
    un0 = ref.get_state(P.FIELD_UN).astype(cdt)
    dev = torch.device("cuda", 0)
    u = torch.from_numpy(u0.copy()).to(dev)
    un = torch.from_numpy(un0.copy()).to(dev)
    params = P.default_params(n=n, precision=prec, viscos=nu, cfl=-1.0, dt=dt, kshift=4)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    for gsh in GSHS:   # two RK steps = two calls of each stage, in a row
        vm_ref = ref.rk_stage(1, gsh, dt=dt)
        ref.rk_stage(2, gsh)
        vm = P.rk_stage_noalloc(params, 1, gsh, dt, u.data_ptr(), un.data_ptr(), stream)
        P.rk_stage_noalloc(params, 2, gsh, dt, u.data_ptr(), un.data_ptr(), stream)
        torch.cuda.synchronize()
        assert abs(vm - vm_ref) <= tol * vm_ref
        assert _rel(un.cpu().numpy(), ref.get_state(P.FIELD_UN)) < tol
        assert _rel(u.cpu().numpy(), ref.get_state(P.FIELD_U)) < tol
    ref.close()


_FRESH = r"""
import sys
import numpy as np
sys.path[:0] = [{root!r}, {pkg!r}]
import torch
import psdns_gpu as P
from oracle import oracle
n, nu, dt = 32, 0.01, 0.004
gshs = {gshs!r}
o = oracle.Oracle(n, nu, cfl=-1, dt=dt, kshift=4)
un0 = o.field_init(77)
o.set_state(un0)
# no Solver (no context, no library allocation) exists in this process
u = torch.from_numpy(un0.copy()).cuda()
un = torch.from_numpy(un0.copy()).cuda()
params = P.default_params(n=n, precision=P.PREC_FP64, viscos=nu, cfl=-1.0, dt=dt, kshift=4)
worst = 0.0
for g in gshs:
    g = np.array(g)
    o.set_shifts(g)
    assert o.stage(1) == 0 and o.stage(2) == 0
    vm = P.rk_stage_noalloc(params, 1, g, dt, u.data_ptr(), un.data_ptr(), 0)
    P.rk_stage_noalloc(params, 2, g, dt, u.data_ptr(), un.data_ptr(), 0)
    torch.cuda.synchronize()
    vo = o.scalars()["velmax"]
    assert abs(vm - vo) <= 1e-12 * vo, (vm, vo)
    uo, uno = o.get_state()
    for got, want in ((un, uno), (u, uo)):
        g_ = got.cpu().numpy()
        worst = max(worst, float(np.linalg.norm(g_ - want) / np.linalg.norm(want)))
assert worst < 1e-11, worst
print("fresh-process noalloc ok", worst)
"""


def test_noalloc_first_call_in_a_fresh_process(gpu_mod, oracle_mod):
    """The real use case: no context was ever created in the process; the
    entry point's own set-up (symbol lookup, tables) runs on the first call."""
    code = _FRESH.format(root=ROOT, pkg=os.path.join(ROOT, "nasa-bluewater-psdns-benchmark-minsky_b200"),
                         gshs=[g.tolist() for g in GSHS])
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process noalloc ok" in r.stdout


def test_noalloc_rejects_boxes_beyond_its_scratch(gpu_mod):
    import torch
    P = gpu_mod
    n = 128
    params = P.default_params(n=n, precision=P.PREC_FP32, viscos=0.01, cfl=-1.0, dt=0.004, kshift=4)
    x = torch.zeros(8, device="cuda")
    with pytest.raises(P.PsdnsError, match="exceeds the largest box"):
        P.rk_stage_noalloc(params, 1, np.zeros((3, 2)), 0.004, x.data_ptr(), x.data_ptr(), 0)


def test_noalloc_rejects_host_memory_and_captured_streams(gpu_mod):
    import torch
    P = gpu_mod
    n = 16
    params = P.default_params(n=n, precision=P.PREC_FP64, viscos=0.01, cfl=-1.0, dt=0.004, kshift=4)
    host = np.zeros((3, 1, n), np.complex128)
    dev = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(P.PsdnsError, match="device"):
        P.rk_stage_noalloc(params, 1, np.zeros((3, 2)), 0.004, host.ctypes.data, dev.data_ptr(), 0)
    # a stream under capture is refused before anything is enqueued on it
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    err = None
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            P.rk_stage_noalloc(params, 1, np.zeros((3, 2)), 0.004, dev.data_ptr(), dev.data_ptr(), s.cuda_stream)
        except P.PsdnsError as e:
            err = str(e)
        dev.add_(1.0)   # the capture stays valid after the refusal
        g.capture_end()
    assert err is not None and "captured" in err
    g.replay()
    torch.cuda.synchronize()
    assert float(dev[0]) == 1.0
