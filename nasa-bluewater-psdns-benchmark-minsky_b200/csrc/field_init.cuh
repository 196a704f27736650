// field_init.cuh -- random solenoidal initial field on the device.
//
// Restates homogeneous/field.f:169-257 (the branch that draws phases with
// ranu, PSDNS/ranu.f) followed by the kx = 0 conjugate symmetry of
// homogeneous/consym.f:35-73.  The reference draws three uniform numbers per
// retained mode in the order of the cylinder traversal (a outer, y inner).
// The generator s_{k+1} = 65539 s_k mod 2^31 (ranu.f:27-28: 32-bit wrap, then
// the sign bit cleared) admits jump-ahead, s_k = s_0 65539^k mod 2^31, so every
// mode computes its own three draws from its position in that order and the
// field is identical to the sequential one.
// Spectrum: E(k) = c0 k^4 exp(-2 (k/3)^2), c0 = 4/(sqrt(pi) 4.5^2.5), whose
// integral is 3/2 (u' = 1).
#pragma once
#include "stage_kernels.cuh"

namespace psdns {

__device__ __forceinline__ uint32_t lcg_jump(uint32_t seed, unsigned long long k) {
  // seed * 65539^k mod 2^31
  unsigned long long r = 1, b = 65539ull;
  const unsigned long long M = 0x7fffffffull;
  while (k) {
    if (k & 1ull) r = (r * b) & M;
    b = (b * b) & M;
    k >>= 1;
  }
  return (uint32_t)(((unsigned long long)seed * r) & M);
}

__device__ __forceinline__ double ranu_at(uint32_t seed, unsigned long long d) {
  // value returned by the (d+1)-th call of ranu after seeding
  return (double)lcg_jump(seed, d + 1) * 0.46566127e-9;
}

template <typename T>
__global__ void k_field_init(Geo g, const long long* __restrict__ off, uint32_t seed, double s1, double s2, double s3,
                             C2<T>* __restrict__ un, C2<T>* __restrict__ u) {
  const int n = g.n;
  const size_t vs = (size_t)g.xz_tot * n;
  const double pi = 3.14159265358979323846;
  const double c0 = 4.0 / (sqrt(pi) * pow(4.5, 2.5));
  const double twopi = 2. * pi, rpid = 1. / sqrt(twopi);
  const double voljac = s1 * s2 * s3;
  const double s1d = 1. / s1, s2d = 1. / s2, s3d = 1. / s3;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < vs; i += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(i / n), y = (int)(i % n);
    C2<T> r1 = cmk<C2<T>>(0, 0), r2 = r1, r3 = r1;
    const int kym = __ldg(g.kymax + a);
    const int km = kym < n / 2 - 1 ? kym : n / 2 - 1;
    const bool inside = (y != n / 2) && (y <= km || y >= n - km);
    if (inside && !(a == 0 && y == 0)) {
      const long long idx = (y <= km ? y : km + 1 + (y - (n - km))) - (a == 0 ? 1 : 0);
      const unsigned long long d = 3ull * (unsigned long long)(off[a] + idx);
      const int x = __ldg(g.ax + a), z = __ldg(g.az + a);
      const double k1u = s1 * x, k3u = s3 * (z > n / 2 ? z - n : z), k2u = s2 * (y > n / 2 ? y - n : y);
      const double kyzsq = k2u * k2u + k3u * k3u;
      const double k = sqrt(k1u * k1u + kyzsq);
      const double kd = 1. / k;
      const double q = k / 3.0;
      const double ekx = c0 * k * k * k * k * exp(-2.0 * q * q) * voljac;
      const double ef = sqrt(ekx) * rpid * kd;
      const double th1 = ranu_at(seed, d), th2 = ranu_at(seed, d + 1), phi = ranu_at(seed, d + 2);
      const double k12 = sqrt(k1u * k1u + k2u * k2u);
      const double ang = twopi * phi, t1 = twopi * th1, t2 = twopi * th2;
      const double ca = cos(ang), sa = sin(ang);
      const double ar = ca * (ef * cos(t1)), ai = ca * (ef * sin(t1));
      const double br = sa * (ef * cos(t2)), bi = sa * (ef * sin(t2));
      if (k12 == 0.) {
        r1 = cmk<C2<T>>((T)(ar / s1), (T)(ai / s1));
        r2 = cmk<C2<T>>((T)(br / s2), (T)(bi / s2));
      } else {
        const double c1r = k * ar, c1i = k * ai, c2r = k3u * br, c2i = k3u * bi;
        const double rt = kd / k12;
        r1 = cmk<C2<T>>((T)(s1d * (rt * (k2u * c1r + k1u * c2r))), (T)(s1d * (rt * (k2u * c1i + k1u * c2i))));
        r2 = cmk<C2<T>>((T)(s2d * (rt * (k2u * c2r - k1u * c1r))), (T)(s2d * (rt * (k2u * c2i - k1u * c1i))));
        r3 = cmk<C2<T>>((T)(-(s3d * (kd * (k12 * br)))), (T)(-(s3d * (kd * (k12 * bi)))));
      }
    }
    un[i] = r1; un[vs + i] = r2; un[2 * vs + i] = r3;
    u[i] = r1; u[vs + i] = r2; u[2 * vs + i] = r3;
  }
}

// consym.f (FRESH): in the kx = 0 plane, u(0,-ky,-kz) = conj(u(0,ky,kz)).
// Columns j = kc0+1 .. 2 kc0 of x = 0 hold kz = j - (2 kc0 + 1) < 0.
template <typename T>
__global__ void k_field_consym(int n, int kc0, int xz_tot, C2<T>* __restrict__ un, C2<T>* __restrict__ u) {
  const size_t vs = (size_t)xz_tot * n;
  const int total = (kc0 + 1) * n;   // column 0 (kz = 0, negative ky) + kc0 negative-kz columns
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * total; i += gridDim.x * blockDim.x) {
    const int v = i / total, r = i % total, jj = r / n, y = r % n;
    C2<T>* U = un + v * vs;
    C2<T>* W = u + v * vs;
    if (jj == 0) {
      if (y > n / 2) {
        const C2<T> s = U[n - y];
        U[y] = cconj(s);
        W[y] = cconj(s);
      }
    } else {
      const int j = kc0 + jj;              // negative kz column
      const int kz = j - (2 * kc0 + 1), jo = -kz;
      const C2<T> s = U[(size_t)jo * n + (y == 0 ? 0 : n - y)];
      U[(size_t)j * n + y] = cconj(s);
      W[(size_t)j * n + y] = cconj(s);
    }
  }
}

}  // namespace psdns
