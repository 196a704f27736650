"""Tensor-core (tcgen05) DFT stage of the mixed-precision arm, through the
C-ABI: the operand layouts on one MMA tile against a float64 product of the
same BF16-rounded operands (tolerance 1e-5 relative: FP32 accumulation of 64
exact products), and the 1024-point line DFT against numpy's float64 FFT of
the same inputs (split-BF16, three products: 3e-5 relative L2; the FP32
Stockham passes: 1e-6)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16_round(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("a_mn_major", [1, 0])
def test_tc_gemm_operand_layouts(gpu_mod, a_mn_major):
    rng = np.random.default_rng(7 + a_mn_major)
    a = bf16_round(rng.standard_normal((128, 64)))
    b = bf16_round(rng.standard_normal((64, 64)))
    d = gpu_mod.tc_gemm_check(a, b, a_mn_major)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    err = np.abs(d - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


@pytest.mark.parametrize("mode,tol", [(1, 3e-5), (0, 1e-6)])
def test_dft_lines_against_numpy(gpu_mod, mode, tol):
    rng = np.random.default_rng(11)
    x = rng.standard_normal((61, 1024)) + 1j * rng.standard_normal((61, 1024))
    x = x.astype(np.complex64).astype(np.complex128)
    got = gpu_mod.dft_lines(x, mode)
    ref = np.fft.fft(x, axis=-1)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    per_line = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    print(f"dft_lines mode {mode}: relative L2 {err:.2e}, worst line {per_line.max():.2e}")
    assert err < tol and per_line.max() < 2 * tol
