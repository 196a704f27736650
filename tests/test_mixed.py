"""The mixed-precision arm: the RK2 step at 1024^3 with every 1-D transform
of the five stage kernels on the tensor cores (PSDNS_DFT_TC_BF16X3:
split-BF16 operands, three products, FP32 accumulation), against the FP64
device step of the same seed (which matches the FP64 oracle to 1e-11 at
256^3, tests/test_accuracy.py) and beside the plain FP32 step.

Tolerances after two forced steps: plain FP32 velocity 1e-6 relative L2;
tensor-core form 1e-4 relative L2, and 1e-4 relative E(k) in the shells
holding at least 1e-6 of the peak (the split-BF16 DFT alone is 4.5e-6 per
transform, tests/test_tc_dft.py)."""
import math

import numpy as np
import pytest


def params(P, n, prec, dft):
    kmax = math.sqrt(2.0) * n / 3.0
    nu = (1.5 / kmax) ** (4.0 / 3.0) * 0.1 ** (1.0 / 3.0)
    return P.default_params(n=n, precision=prec, viscos=nu, cfl=math.pi, dt=0.0, kshift=1, kforce=2.99,
                            tforce=0.5, epsfor=0.1 / (4.0 * (4.0 * math.pi / 3.0) * 27.0), tfiuo=0.0, dft=dft)


def test_tensor_core_form_needs_fp32_at_1024(gpu_mod):
    """Refused on the host before any device work (runs without a GPU)."""
    P = gpu_mod
    with pytest.raises(P.PsdnsError, match="FP32 state at n = 1024"):
        P.Solver(params(P, 64, P.PREC_FP32, P.DFT_TC_BF16X3))
    with pytest.raises(P.PsdnsError, match="FP32 state at n = 1024"):
        P.Solver(params(P, 1024, P.PREC_FP64, P.DFT_TC_BF16X3))


@pytest.mark.gpu
def test_mixed_arm_against_fp64_at_1024(gpu_mod):
    P = gpu_mod
    n, steps = 1024, 2
    out = {}
    for name, prec, dft in (("fp64", P.PREC_FP64, P.DFT_FP32), ("fp32", P.PREC_FP32, P.DFT_FP32),
                            ("tc", P.PREC_FP32, P.DFT_TC_BF16X3)):
        s = P.Solver(params(P, n, prec, dft))
        s.field_init(1234)
        for _ in range(steps):
            info = s.step()
            assert info["status"] == 0
        out[name] = (s.get_state(P.FIELD_UN), s.spectra(P.FIELD_UN)[0], info["velmax"])
        s.close()
    ref, ek_ref, vm_ref = out.pop("fp64")
    nrm = np.sqrt(sum(float(np.vdot(ref[v], ref[v]).real) for v in range(3)))
    m = ek_ref > 1e-6 * ek_ref.max()
    errs = {}
    for name, (un, ek, vm) in out.items():
        d2 = sum(float(np.vdot(un[v] - ref[v], un[v] - ref[v]).real) for v in range(3))
        errs[name] = (math.sqrt(d2) / nrm, float(np.max(np.abs(ek[m] - ek_ref[m]) / ek_ref[m])), abs(vm / vm_ref - 1))
        print(f"{name}: velocity rel L2 {errs[name][0]:.2e}, max rel E(k) {errs[name][1]:.2e} "
              f"({int(m.sum())} shells), velmax {errs[name][2]:.2e}")
    assert errs["fp32"][0] < 1e-6
    assert errs["tc"][0] < 1e-4
    assert errs["tc"][1] < 1e-4
    assert errs["tc"][2] < 1e-4
