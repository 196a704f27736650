// spectra.cuh -- FP64 shell spectra of the velocity state on the device.
//
// Restates homogeneous/sptr.f:139-193 (per-mode products tfact*Re(u_i u_j*)
// binned by shell ik = int(|k| + 1.5), dissipation and skewness moments scaled
// by 2 nu, :235-237) and the derived statistics of :350-400 (E(k), D(k), TKE,
// epsilon, spectral derivative skewness, Kolmogorov scales, integral scale).
// All accumulation is FP64 whatever the state precision: each block keeps
// shell histograms in shared memory (FP64 shared atomics) and adds them to
// the global sums once.
#pragma once
#include "stage_kernels.cuh"

namespace psdns {

// per shell: E_ij (6: 11,12,13,22,23,33), D_ii sum, S_ii sum, ekk
constexpr int kSpecVals = 9;

// One warp per column (kx, kz); lane l takes the contiguous y run
// [l c, l c + c), c = ceil(n / 32), so that its shell index changes only a
// few times along the run: the nine sums of the current shell stay in
// registers and go to the shared histogram (FP64 shared atomics) when the
// shell changes.  A warp load reads 32 sectors, one per lane, whose other
// bytes the lane's next loads take from L1.  (One thread per mode, with nine
// shared atomics per mode on the few shells a warp's consecutive y share,
// ran at 4% of the DRAM bandwidth, held at the block barrier.)
template <typename T>
__global__ void __launch_bounds__(512) k_spectra(Geo g, const C2<T>* __restrict__ un, double b11, double b22,
                                                 double b33, int nshell, double* __restrict__ out) {
  extern __shared__ double hist[];   // [nshell][kSpecVals]
  const int n = g.n;
  for (int i = threadIdx.x; i < nshell * kSpecVals; i += blockDim.x) hist[i] = 0.0;
  __syncthreads();
  const size_t vs = (size_t)g.xz_tot * n;
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  const int run = (n + 31) / 32, y0 = min(lane * run, n), y1 = min(y0 + run, n);
  for (int a = blockIdx.x * warps + (threadIdx.x >> 5); a < g.xz_tot; a += gridDim.x * warps) {
    const int x = __ldg(g.ax + a), z = __ldg(g.az + a), km = __ldg(g.kymax + a);
    const double kx = x, kz = z > n / 2 ? z - n : z;
    const double tf = x == 0 ? 1.0 : 2.0;
    const double rxz = b11 * kx * kx + b33 * kz * kz;
    double acc[kSpecVals];
    int cur = -1;
    auto flush = [&]() {
      if (cur >= 0) {
        double* h = hist + cur * kSpecVals;
#pragma unroll
        for (int v = 0; v < kSpecVals; v++)
          if (acc[v] != 0.0) atomicAdd(h + v, acc[v]);
      }
    };
    for (int y = y0; y < y1; y++) {
      // masks.f: y != n/2 and min(y, n - y) <= kymax(a)
      const int kya = y > n / 2 ? n - y : y;
      if (y == n / 2 || kya > km) continue;
      const double ky = y > n / 2 ? y - n : y;
      // sptr.f:85-97: Nyquist rows contribute no wavenumber (masked anyway)
      const double rk2 = rxz + b22 * ky * ky, rk = sqrt(rk2);
      const int ik = (int)(rk + 1.5) - 1;
      if (ik < 0 || ik >= nshell) continue;
      if (ik != cur) {
        flush();
        cur = ik;
#pragma unroll
        for (int v = 0; v < kSpecVals; v++) acc[v] = 0.0;
      }
      const size_t i = (size_t)a * n + y;
      const C2<T> u1 = un[i], u2 = un[vs + i], u3 = un[2 * vs + i];
      const double a1 = u1.x, c1 = u1.y, a2 = u2.x, c2 = u2.y, a3 = u3.x, c3 = u3.y;
      const double e11 = tf * (a1 * a1 + c1 * c1), e22 = tf * (a2 * a2 + c2 * c2), e33 = tf * (a3 * a3 + c3 * c3);
      acc[0] += e11;
      acc[1] += tf * (a1 * a2 + c1 * c2);
      acc[2] += tf * (a1 * a3 + c1 * c3);
      acc[3] += e22;
      acc[4] += tf * (a2 * a3 + c2 * c3);
      acc[5] += e33;
      const double tr = e11 + e22 + e33;
      acc[6] += rk2 * tr;
      acc[7] += rk2 * rk2 * tr;
      if (rk2 != 0.) acc[8] += (e11 * b11 + e22 * b22 + e33 * b33) / rk;
    }
    flush();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nshell * kSpecVals; i += blockDim.x)
    if (hist[i] != 0.0) atomicAdd(out + i, hist[i]);
}

// One-dimensional spectra and the derivative variance of sptr.f:119-218 for
// the 6 velocity products ij (11,12,13,22,23,33): per column a (kx, kz) the
// y-sum of Re(u_i u_j*) over the sphere goes to xr[ij][kx] and to
// zr[ij][|kz|] (conjugate-symmetric halves folded as sptr.f:198-205), each
// mode to yr[ij][|ky|] (:150-159), and ky2 Re(u_i u_j*) tfact to der2[ij].
// out layout: xr[6][n/2+1], yr[6][n/2+1], zr[6][n/2+1], der2[6].  One warp
// per column; shared-memory FP64 histograms, added to out once per block.
constexpr int kSpec1dPairs = 6;

template <typename T>
__global__ void __launch_bounds__(512) k_spectra_1d(Geo g, const C2<T>* __restrict__ un, double b22,
                                                    double* __restrict__ out) {
  extern __shared__ double h1[];
  const int n = g.n, nh = n / 2 + 1;
  const int nv = 3 * kSpec1dPairs * nh + kSpec1dPairs;
  for (int i = threadIdx.x; i < nv; i += blockDim.x) h1[i] = 0.0;
  __syncthreads();
  double* xr = h1;
  double* yr = h1 + kSpec1dPairs * nh;
  double* zr = h1 + 2 * kSpec1dPairs * nh;
  double* d2 = h1 + 3 * kSpec1dPairs * nh;
  const size_t vs = (size_t)g.xz_tot * n;
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  double der2[kSpec1dPairs] = {0, 0, 0, 0, 0, 0};
  for (int a = blockIdx.x * warps + (threadIdx.x >> 5); a < g.xz_tot; a += gridDim.x * warps) {
    const int x = __ldg(g.ax + a), z = __ldg(g.az + a), km = __ldg(g.kymax + a);
    const double tf = x == 0 ? 1.0 : 2.0;
    double ysum[kSpec1dPairs] = {0, 0, 0, 0, 0, 0};
    for (int y = lane; y < n; y += 32) {
      const int ky = y > n / 2 ? n - y : y;
      if (y == n / 2 || ky > km) continue;
      const size_t o = (size_t)a * n + y;
      const C2<T> u1 = un[o], u2 = un[vs + o], u3 = un[2 * vs + o];
      const double a1 = u1.x, c1 = u1.y, a2 = u2.x, c2 = u2.y, a3 = u3.x, c3 = u3.y;
      const double p[kSpec1dPairs] = {a1 * a1 + c1 * c1, a1 * a2 + c1 * c2, a1 * a3 + c1 * c3,
                                      a2 * a2 + c2 * c2, a2 * a3 + c2 * c3, a3 * a3 + c3 * c3};
      const double ky2 = b22 * (double)ky * (double)ky;
#pragma unroll
      for (int ij = 0; ij < kSpec1dPairs; ij++) {
        ysum[ij] += p[ij];
        der2[ij] += ky2 * (tf * p[ij]);
        if (y == 0) atomicAdd(yr + ij * nh, tf * p[ij]);
        else if (y < n / 2) atomicAdd(yr + ij * nh + y, p[ij]);
        else if (tf > 1.0) atomicAdd(yr + ij * nh + (n - y), p[ij]);
      }
    }
#pragma unroll
    for (int ij = 0; ij < kSpec1dPairs; ij++) {
      double v = ysum[ij];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) {
        atomicAdd(xr + ij * nh + x, v);
        if (z == 0) atomicAdd(zr + ij * nh, tf * v);
        else if (z < n / 2) atomicAdd(zr + ij * nh + z, v);
        else if (z > n / 2 && tf > 1.0) atomicAdd(zr + ij * nh + (n - z), v);
      }
    }
  }
#pragma unroll
  for (int ij = 0; ij < kSpec1dPairs; ij++) {
    double v = der2[ij];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(d2 + ij, v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nv; i += blockDim.x)
    if (h1[i] != 0.0) atomicAdd(out + i, h1[i]);
}

}  // namespace psdns
