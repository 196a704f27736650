"""psdns_gpu_rk_stage_noalloc: the RK stage for callers that cannot call
cudaMalloc (for instance a driver whose device arrays belong to another
runtime, or one with a fixed device-memory budget).  It runs on the caller's
own device arrays with its scratch in a static device array, and must give the
same result as the context-based psdns_gpu_rk_stage.

Collected last on purpose (file name), so that a run stopping at the first
failure has already run every other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("n", [32, 64])
def test_noalloc_stage_matches_context_stage(gpu_mod, n):
    import torch
    P = gpu_mod
    nu, dt = 0.01, 0.004
    ref = P.Solver(n=n, precision=P.PREC_FP64, viscos=nu, cfl=-1.0, dt=dt, kshift=4)
    ref.field_init(31 + n)
    u0 = ref.get_state(P.FIELD_U)
    un0 = ref.get_state(P.FIELD_UN)
    dev = torch.device("cuda", 0)
    u = torch.from_numpy(u0.copy()).to(dev)
    un = torch.from_numpy(un0.copy()).to(dev)
    params = P.default_params(n=n, precision=P.PREC_FP64, viscos=nu, cfl=-1.0, dt=dt, kshift=4)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    gshs = [np.array([[0.1, 0.6], [0.3, 0.8], [0.45, 0.95]]), np.array([[0.7, 0.2], [0.05, 0.55], [0.9, 0.4]])]
    for gsh in gshs:   # two RK steps = two calls of each stage, in a row
        vm_ref = ref.rk_stage(1, gsh, dt=dt)
        ref.rk_stage(2, gsh)
        vm = P.rk_stage_noalloc(params, 1, gsh, dt, u.data_ptr(), un.data_ptr(), stream)
        P.rk_stage_noalloc(params, 2, gsh, dt, u.data_ptr(), un.data_ptr(), stream)
        torch.cuda.synchronize()
        assert abs(vm - vm_ref) <= 1e-12 * vm_ref
        assert _rel(un.cpu().numpy(), ref.get_state(P.FIELD_UN)) < 1e-12
        assert _rel(u.cpu().numpy(), ref.get_state(P.FIELD_U)) < 1e-12
    ref.close()


def test_noalloc_rejects_boxes_beyond_its_scratch(gpu_mod):
    import torch
    P = gpu_mod
    n = 128
    params = P.default_params(n=n, precision=P.PREC_FP32, viscos=0.01, cfl=-1.0, dt=0.004, kshift=4)
    x = torch.zeros(8, device="cuda")
    with pytest.raises(P.PsdnsError, match="exceeds the largest box"):
        P.rk_stage_noalloc(params, 1, np.zeros((3, 2)), 0.004, x.data_ptr(), x.data_ptr(), 0)
