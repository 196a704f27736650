// learned.cuh -- device kernels of the learned coarse solver that act on a
// box's state: the spectral filter that makes a coarse box from a fine one
// (the training and evaluation data), and the per-shell damping through which
// the spectral-correction network (learned.cu) acts on the coarse state.
#pragma once
#include "stage_kernels.cuh"

namespace psdns {

// Coarse u and un = the modes of the fine un that lie inside the coarse
// box's truncation sphere (a sharp filter in wavenumber space: the Fourier
// coefficients are those of the physical field, independent of n, so they
// are copied as they are).  Coarse entries outside the sphere are zero.
// Element (v, a, y) of the coarse YCYL array per thread, grid-stride.
template <typename T>
__global__ void __launch_bounds__(256) k_filter_state(Geo gf, const C2<T>* __restrict__ fin, Geo gc,
                                                      C2<T>* __restrict__ u, C2<T>* __restrict__ un) {
  using C = C2<T>;
  const size_t per = (size_t)gc.xz_tot * gc.n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < 3 * per; e += (size_t)gridDim.x * blockDim.x) {
    const int v = (int)(e / per);
    const size_t r = e % per;
    const int a = (int)(r / gc.n), y = (int)(r % gc.n);
    C val = cmk<C>(0, 0);
    if (mask_ok(gc, a, y, gc.n)) {
      const int x = __ldg(gc.ax + a), zc = __ldg(gc.az + a);
      const int kz = zc > gc.n / 2 ? zc - gc.n : zc;
      const int ky = y > gc.n / 2 ? y - gc.n : y;
      const int c0 = __ldg(gf.colstart + x), kcf = (__ldg(gf.colstart + x + 1) - c0 - 1) / 2;
      if (x < gf.kxn && kz <= kcf && -kz <= kcf) {
        // fine column x holds kz = 0..kcf then -kcf..-1 (mpisetup.f:322-357)
        const int af = c0 + (kz >= 0 ? kz : 2 * kcf + 1 + kz);
        const int yf = ky >= 0 ? ky : gf.n + ky;
        val = fin[((size_t)v * gf.xz_tot + af) * gf.n + yf];
      }
    }
    u[e] = val;
    un[e] = val;
  }
}

// u and un (velocity) of every mode whose shell index int(|k| + 0.5) is in
// 1 .. nshell are multiplied by f[shell] (f[0] unused)
template <typename T>
__global__ void __launch_bounds__(256) k_shell_factor(Geo g, C2<T>* __restrict__ u, C2<T>* __restrict__ un,
                                                      const double* __restrict__ f, int nshell, double b11,
                                                      double b22, double b33) {
  const size_t per = (size_t)g.xz_tot * g.n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < 3 * per; e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e % per;
    const int a = (int)(r / g.n), y = (int)(r % g.n);
    const int x = __ldg(g.ax + a), z = __ldg(g.az + a);
    const int ky = y > g.n / 2 ? y - g.n : y, kz = z > g.n / 2 ? z - g.n : z;
    const double k = sqrt(b11 * x * x + b22 * ky * ky + b33 * kz * kz);
    const int sh = (int)(k + 0.5);
    if (sh >= 1 && sh <= nshell) {
      const T s = (T)__ldg(f + sh);
      u[e] = cscale(s, u[e]);
      un[e] = cscale(s, un[e]);
    }
  }
}

}  // namespace psdns
