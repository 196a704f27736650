"""Host-side model of the register-level pair packing of the x chain
(csrc/stage_kernels.cuh: XFuse, xchain_load_pass0, xchain_last_store).

For the two-pass FP32 plans of fft_core.cuh (plan_rad: R0 = 2^(K/2),
R1 = 2^(K - K/2), E = lcm(R0, R1), P = N / E) lane t of a line holds the
elements t + P m both as pass-0 operands and as last-pass outputs, and the
Hermitian partner N - x of its element x sits in lane (P - t) mod P.  The
model below replays the kernels' per-lane arithmetic (loads of A(x), B(x)
for x < N/2, one shuffle per slot, lane 0's own slots) and checks it against
the packed line that xchain_pack writes through shared memory, and the
unpacking against xchain_store.  No GPU is needed."""
import numpy as np
import pytest


def plan_fp32(n):
    k = n.bit_length() - 1
    if k <= 3:
        return [n]
    return [1 << (k // 2), 1 << (k - k // 2)]


def kxn_of(n):
    return min(n // 2, int(n * 2 ** 0.5 / 3) + 1)


def packed_line(a, b, n, kxn):
    """The line xchain_pack writes: conj(A + iB) with the Hermitian half."""
    z = np.zeros(n, complex)
    z[0] = complex(a[0].real, -b[0].real)
    for x in range(1, kxn):
        z[x] = complex(a[x].real - b[x].imag, -(a[x].imag + b[x].real))
        z[n - x] = complex(a[x].real + b[x].imag, -(b[x].real - a[x].imag))
    return z


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512, 1024])
def test_lane_model_of_pair_packing(n):
    r0, r1 = plan_fp32(n)
    e = max(r0, r1)
    p = n // e
    h = r1 // 2
    nb = e // r0
    # the XFuse conditions: two passes, last radix = operands per thread
    assert r1 == e and p == r0 and 32 % p == 0
    rng = np.random.default_rng(n)
    for kxn in sorted({kxn_of(n), n // 2, 3}):
        a = rng.standard_normal(kxn) + 1j * rng.standard_normal(kxn)
        b = rng.standard_normal(kxn) + 1j * rng.standard_normal(kxn)
        want = packed_line(a, b, n, kxn)
        # loads: lane t, slot m < H, x = t + P m
        av = np.zeros((p, h), complex)
        bv = np.zeros((p, h), complex)
        for t in range(p):
            for m in range(h):
                x = t + p * m
                if x < kxn:
                    av[t, m], bv[t, m] = a[x], b[x]
        zl = np.zeros((p, r1), complex)
        for m in range(h):
            mv = np.array([complex(av[t, m].real + bv[t, m].imag, -(bv[t, m].real - av[t, m].imag))
                           for t in range(p)])
            for t in range(p):
                aa, bb = av[t, m], bv[t, m]
                zl[t, m] = (complex(aa.real, -bb.real) if (t == 0 and m == 0)
                            else complex(aa.real - bb.imag, -(aa.imag + bb.real)))
                got = mv[(p - t) & (p - 1)]     # __shfl_sync(.., src = (P - t) & (P - 1), P)
                if t != 0:
                    zl[t, r1 - 1 - m] = got
                elif m >= 1:
                    zl[t, r1 - m] = mv[t]
        for t in range(p):
            for m in range(r1):
                assert zl[t, m] == pytest.approx(want[t + p * m], abs=1e-12)
            # pass-0 operand order: butterfly q, operand r is element t + q P + r (N / R0)
            for q in range(nb):
                for r in range(r0):
                    assert t + q * p + r * (n // r0) == t + p * (q + nb * r)
        # unpacking: lane t holds Y(t + P m) after the last pass
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        v = np.array([[y[t + p * m] for m in range(r1)] for t in range(p)])
        stored = {}
        for m in range(h):
            sent = v[:, r1 - 1 - m]
            for t in range(p):
                yn = v[t, (r1 - m) % r1] if t == 0 else sent[(p - t) & (p - 1)]
                x = t + p * m
                assert yn == y[(n - x) % n]
                if x < kxn:
                    stored[x] = stored.get(x, 0) + 1
        assert sorted(stored) == list(range(kxn)) and set(stored.values()) == {1}
