// fft_core.cuh -- batched 1-D complex FFT of lines held in shared memory.
//
// Replaces the FFTW 1-D transforms the reference plans in PSDNS/epfftw.f
// (plan4_p1/plan4_p3 along y, plan2_kx/plan2_xk along z, plan3_p2c/plan1_p2b
// along x).  Unnormalised forward transform X_k = sum_j x_j exp(-2 pi i jk/N);
// the backward transform is obtained by conjugating input and output.
//
// Algorithm: Stockham auto-sort with mixed register radices.  A line of N
// points is split into passes of radix R_p (product = N).  In every pass each
// thread owns E/R_p butterflies of radix R_p whose operands it holds in
// registers; the radix-R kernels are unrolled at compile time with constant
// twiddles.  Between passes data goes through shared memory in place: all
// operands are read, the block synchronises, then all results are written.
// Shared-memory element i of a line lives at pad(i) = i + i/32, which keeps
// the strided writes of the first pass from serialising on one bank.  The
// inter-pass twiddles of pass p are stored as a table [r][k] (k = j mod Ns)
// so that consecutive threads read consecutive words.
#pragma once
#include <type_traits>
#include <cuda_runtime.h>
#include <stdint.h>

namespace psdns {

template <typename T> struct V2;
template <> struct V2<float> { using type = float2; };
template <> struct V2<double> { using type = double2; };
template <typename T> using C2 = typename V2<T>::type;

template <typename C> struct ElemOf;
template <> struct ElemOf<float2> { using type = float; };
template <> struct ElemOf<double2> { using type = double; };

template <typename C>
__host__ __device__ __forceinline__ C cmk(typename ElemOf<C>::type a, typename ElemOf<C>::type b) {
  C r; r.x = a; r.y = b; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmk<C>(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cscale(typename ElemOf<C>::type s, C a) {
  return cmk<C>(s * a.x, s * a.y);
}
// multiply by -i (forward quarter turn)
template <typename C> __device__ __forceinline__ C cmul_mi(C a) { return cmk<C>(a.y, -a.x); }
// multiply by +i
template <typename C> __device__ __forceinline__ C cmul_pi(C a) { return cmk<C>(-a.y, a.x); }

// ---------------------------------------------------------------------------
// Compile-time cos/sin of 2*pi*k/R (Taylor series on a quadrant-reduced
// argument |phi| <= pi/4; exact to double rounding for the radices used).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr double ct_sin_small(double x) {
  double x2 = x * x, term = x, sum = x;
  for (int n = 1; n < 14; n++) { term = -term * x2 / double((2 * n) * (2 * n + 1)); sum += term; }
  return sum;
}
__host__ __device__ constexpr double ct_cos_small(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int n = 1; n < 14; n++) { term = -term * x2 / double((2 * n - 1) * (2 * n)); sum += term; }
  return sum;
}
// returns cos(2 pi k / R) (which = 0) or sin(2 pi k / R) (which = 1)
__host__ __device__ constexpr double ct_trig(int k, int R, int which) {
  int m = ((k % R) + R) % R;
  // 4m/R = q + f with q the nearest quadrant, |f| <= 1/2
  long num = 4L * m;            // angle = (num / R) * (pi/2)
  long q = (2 * num + R) / (2 * R);   // round(num / R)
  double f = double(num - q * R) / double(R);   // in [-1/2, 1/2]
  double phi = f * 1.57079632679489661923;
  double c = ct_cos_small(phi), s = ct_sin_small(phi);
  int qq = int(q % 4);
  double cc = 0, ss = 0;
  if (qq == 0) { cc = c; ss = s; }
  else if (qq == 1) { cc = -s; ss = c; }
  else if (qq == 2) { cc = -c; ss = -s; }
  else { cc = s; ss = -c; }
  return which == 0 ? cc : ss;
}

// multiply o by W_R^K = exp(-2 pi i K / R) with compile-time constants
template <int K, int R, typename C>
__device__ __forceinline__ C tw_const(C o) {
  using T = typename ElemOf<C>::type;
  constexpr int k = ((K % R) + R) % R;
  if constexpr (k == 0) {
    return o;
  } else if constexpr (4 * k == R) {
    return cmul_mi(o);
  } else if constexpr (2 * k == R) {
    return cmk<C>(-o.x, -o.y);
  } else if constexpr (4 * k == 3 * R) {
    return cmul_pi(o);
  } else if constexpr (8 * k == R) {
    constexpr T h = T(0.70710678118654752440);
    return cmk<C>((o.x + o.y) * h, (o.y - o.x) * h);
  } else if constexpr (8 * k == 3 * R) {
    constexpr T h = T(0.70710678118654752440);
    return cmk<C>((o.y - o.x) * h, -(o.x + o.y) * h);
  } else {
    constexpr T cr = T(ct_trig(k, R, 0));
    constexpr T ci = T(-ct_trig(k, R, 1));
    return cmk<C>(o.x * cr - o.y * ci, o.x * ci + o.y * cr);
  }
}

// ---------------------------------------------------------------------------
// In-register DFT of R points v[0], v[S], ..., v[(R-1)S] (natural order in
// and out), forward sign.  Radix-2 decimation in time, radix-4 and radix-3
// leaves.
// ---------------------------------------------------------------------------
template <int R, int S, typename C> __device__ __forceinline__ void dft_s(C* v);

template <int K, int R, int S, typename C>
__device__ __forceinline__ void dit2_combine(C* v, C* tmp) {
  if constexpr (K < R / 2) {
    C e = v[2 * S * K];
    C o = tw_const<K, R>(v[S + 2 * S * K]);
    tmp[K] = cadd(e, o);
    tmp[K + R / 2] = csub(e, o);
    dit2_combine<K + 1, R, S>(v, tmp);
  }
}

template <int K, int R, int S, typename C>
__device__ __forceinline__ void dit3_combine(C* v, C* tmp) {
  using T = typename ElemOf<C>::type;
  if constexpr (K < R / 3) {
    constexpr int M = R / 3;
    C a = v[3 * S * K];
    C b = tw_const<K, R>(v[S + 3 * S * K]);
    C c = tw_const<2 * K, R>(v[2 * S + 3 * S * K]);
    // radix-3 butterfly, W3 = exp(-2 pi i/3) = (-1/2, -sqrt(3)/2)
    constexpr T h = T(0.86602540378443864676);
    C s = cadd(b, c), d = csub(b, c);
    C m = cmk<C>(a.x - T(0.5) * s.x, a.y - T(0.5) * s.y);
    C r = cmk<C>(h * d.y, -h * d.x);   // -i*sqrt(3)/2 * d
    tmp[K] = cadd(a, s);
    tmp[K + M] = cadd(m, r);
    tmp[K + 2 * M] = csub(m, r);
    dit3_combine<K + 1, R, S>(v, tmp);
  }
}

template <int R, int S, typename C>
__device__ __forceinline__ void dft_s(C* v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    C a = v[0], b = v[S];
    v[0] = cadd(a, b);
    v[S] = csub(a, b);
  } else if constexpr (R == 4) {
    C a = v[0], b = v[S], c = v[2 * S], d = v[3 * S];
    C t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = cmul_mi(csub(b, d));
    v[0] = cadd(t0, t2);
    v[2 * S] = csub(t0, t2);
    v[S] = cadd(t1, t3);
    v[3 * S] = csub(t1, t3);
  } else if constexpr (R % 4 == 0 || R % 2 == 0 && R % 3 != 0) {
    dft_s<R / 2, 2 * S>(v);
    dft_s<R / 2, 2 * S>(v + S);
    C tmp[R];
    dit2_combine<0, R, S>(v, tmp);
#pragma unroll
    for (int k = 0; k < R; k++) v[S * k] = tmp[k];
  } else if constexpr (R % 3 == 0) {
    dft_s<R / 3, 3 * S>(v);
    dft_s<R / 3, 3 * S>(v + S);
    dft_s<R / 3, 3 * S>(v + 2 * S);
    C tmp[R];
    dit3_combine<0, R, S>(v, tmp);
#pragma unroll
    for (int k = 0; k < R; k++) v[S * k] = tmp[k];
  } else {
    static_assert(R % 2 == 0 || R % 3 == 0, "unsupported radix");
  }
}

// ---------------------------------------------------------------------------
// Pass plans.  N = R0 * R1 [* R2]; E = max radix (operands per thread),
// P = N / E threads per line.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ilog2c(int n) { int k = 0; while ((1 << k) < n) k++; return k; }

__host__ __device__ constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
__host__ __device__ constexpr int plan_npass(int N, bool dbl) {
  return is_pow2(N) ? ((ilog2c(N) <= 3) ? 1 : ((dbl && ilog2c(N) >= 9) ? 3 : 2)) : 2;
}
__host__ __device__ constexpr int plan_rad(int N, bool dbl, int p) {
  if (is_pow2(N)) {
    const int K = ilog2c(N), np = plan_npass(N, dbl);
    if (np == 1) return p == 0 ? N : 1;
    if (np == 2) return p == 0 ? (1 << (K / 2)) : (p == 1 ? (1 << (K - K / 2)) : 1);
    const int a = (K + 2) / 3, b = (K - a + 1) / 2, c = K - a - b;
    return p == 0 ? (1 << a) : (p == 1 ? (1 << b) : (p == 2 ? (1 << c) : 1));
  }
  if (N == 6) return p == 0 ? 6 : 1;
  if (N == 12) return p == 0 ? 3 : (p == 1 ? 4 : 1);
  if (N == 24) return p == 0 ? 6 : (p == 1 ? 4 : 1);
  if (N == 48) return p == 0 ? 12 : (p == 1 ? 4 : 1);
  if (N == 96) return p == 0 ? 12 : (p == 1 ? 8 : 1);
  return 1;
}
__host__ __device__ constexpr int gcd_i(int a, int b) { return b == 0 ? a : gcd_i(b, a % b); }
// operands per thread: a multiple of every radix (their lcm), so that each
// pass gives every thread whole butterflies
__host__ __device__ constexpr int plan_e(int N, bool dbl) {
  int e = 1;
  for (int p = 0; p < 3; p++) { int r = plan_rad(N, dbl, p); e = e / gcd_i(e, r) * r; }
  return e;
}
__host__ __device__ constexpr int plan_ns(int N, bool dbl, int p) {
  int s = 1; for (int i = 0; i < p; i++) s *= plan_rad(N, dbl, i); return s;
}
// Passes p >= 1 of radix >= 16 (a multiple of 8) keep factored twiddles:
// W^(r k) = W^(8 (r/8) k) * W^((r%8) k), rows [0..7] of W^(r0 k) then rows
// [8 .. 8 + R/8 - 1] of W^(8 r1 k), so a thread loads 8 + R/8 twiddles
// instead of R (radix 32: 12 instead of 32) and forms the rest with one
// complex product each.
__host__ __device__ constexpr bool plan_fact(int N, bool dbl, int p) {
  return p >= 1 && plan_rad(N, dbl, p) >= 16 && plan_rad(N, dbl, p) % 8 == 0;
}
__host__ __device__ constexpr int plan_twsz(int N, bool dbl, int p) {
  return plan_fact(N, dbl, p) ? (8 + plan_rad(N, dbl, p) / 8) * plan_ns(N, dbl, p)
                              : plan_rad(N, dbl, p) * plan_ns(N, dbl, p);
}
__host__ __device__ constexpr int plan_twoff(int N, bool dbl, int p) {
  int o = 0; for (int i = 1; i < p; i++) o += plan_twsz(N, dbl, i); return o;
}

template <typename T, int N> struct FFTPlan {
  static constexpr bool DBL = sizeof(T) == 8;
  static_assert(is_pow2(N) || N == 48 || N == 96 || N == 24 || N == 12 || N == 6,
                "N must be a power of two (or 6*2^k up to 96)");
  static constexpr int NPASS = plan_npass(N, DBL);
  static constexpr int rad(int p) { return plan_rad(N, DBL, p); }
  static constexpr int E = plan_e(N, DBL);
  static constexpr int P = N / E;   // threads per line
  static_assert(P * E == N, "operands per thread must divide the line");
  static constexpr int ns(int p) { return plan_ns(N, DBL, p); }
  static constexpr int twoff(int p) { return plan_twoff(N, DBL, p); }
  static constexpr bool fact(int p) { return plan_fact(N, DBL, p); }
  static constexpr int TWSIZE = plan_twoff(N, DBL, plan_npass(N, DBL)) > 0 ? plan_twoff(N, DBL, plan_npass(N, DBL)) : 1;
};

__host__ __device__ __forceinline__ constexpr int pad32(int i) { return i + (i >> 5); }
template <int N> struct LineLen { static constexpr int value = N + N / 32; };

// Barrier among the threads that share a line.  When a line lives inside one
// warp (P divides 32) a warp barrier suffices; otherwise the whole block
// synchronises.
template <int P>
__device__ __forceinline__ void line_sync() {
  if constexpr (P <= 32 && (32 % P) == 0) {
    __syncwarp();
  } else {
    __syncthreads();
  }
}

// Operands of butterfly set q of thread t in one Stockham pass: read from the
// line, twiddled, transformed in registers (v[q R .. q R + R - 1]).
template <typename C, int N, int R, int NS, int E, int P, bool FACT>
__device__ __forceinline__ void pass_butterflies(const C* line, int t, const C* __restrict__ twp, C* v) {
  constexpr int NB = E / R;
#pragma unroll
  for (int q = 0; q < NB; q++) {
    const int j = t + q * P;
    const int k = j % NS;
#pragma unroll
    for (int r = 0; r < R; r++) v[q * R + r] = line[pad32(j + r * (N / R))];
    if constexpr (FACT) {
      C t0[8];
#pragma unroll
      for (int r0 = 1; r0 < 8; r0++) t0[r0] = twp[r0 * NS + k];
#pragma unroll
      for (int r0 = 1; r0 < 8; r0++) v[q * R + r0] = cmul(v[q * R + r0], t0[r0]);
#pragma unroll
      for (int r1 = 1; r1 < R / 8; r1++) {
        const C t1 = twp[(8 + r1) * NS + k];
        v[q * R + 8 * r1] = cmul(v[q * R + 8 * r1], t1);
#pragma unroll
        for (int r0 = 1; r0 < 8; r0++) v[q * R + 8 * r1 + r0] = cmul(v[q * R + 8 * r1 + r0], cmul(t1, t0[r0]));
      }
    } else if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; r++) v[q * R + r] = cmul(v[q * R + r], twp[r * NS + k]);
    }
    dft_s<R, 1>(v + q * R);
  }
}

// One Stockham pass over nlines lines (rounds of LPR lines).
template <typename C, int N, int R, int NS, int E, int P, int THREADS, bool FACT>
__device__ __forceinline__ void fft_pass(C* buf, int nlines, int ls, const C* __restrict__ twp) {
  constexpr int LPR = THREADS / P;
  constexpr int NB = E / R;   // butterflies per thread
  static_assert(NB * R == E && NB * P * R == N, "a pass must give every thread whole butterflies");
  const int tid = threadIdx.x;
  const int lr = tid / P, t = tid % P;
  for (int l0 = 0; l0 < nlines; l0 += LPR) {
    const int l = l0 + lr;
    const bool act = (lr < LPR) && (l < nlines);
    C v[E];
    C* line = buf + (size_t)l * ls;
    if (act) pass_butterflies<C, N, R, NS, E, P, FACT>(line, t, twp, v);
    line_sync<P>();
    if (act) {
#pragma unroll
      for (int q = 0; q < NB; q++) {
        const int j = t + q * P;
        const int k = j % NS;
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) line[pad32(base + r * NS)] = v[q * R + r];
      }
    }
    line_sync<P>();
  }
}

template <typename T, int N, int THREADS, int PASS>
__device__ __forceinline__ void fft_passes(C2<T>* buf, int nlines, int ls, const C2<T>* tw) {
  using PL = FFTPlan<T, N>;
  if constexpr (PASS < PL::NPASS) {
    constexpr int R = PL::rad(PASS);
    constexpr int NS = PL::ns(PASS);
    fft_pass<C2<T>, N, R, NS, PL::E, PL::P, THREADS, PL::fact(PASS)>(buf, nlines, ls, tw + PL::twoff(PASS));
    fft_passes<T, N, THREADS, PASS + 1>(buf, nlines, ls, tw);
  }
}

// Forward FFT of nlines lines in shared memory (line l at buf + l*ls,
// element i at pad32(i)); tw = shared twiddle table of FFTPlan<T,N>.
// Must be called by all THREADS threads of the block (contains barriers).
template <typename T, int N, int THREADS>
__device__ __forceinline__ void fft_lines(C2<T>* buf, int nlines, int ls, const C2<T>* tw) {
  static_assert(THREADS % FFTPlan<T, N>::P == 0, "THREADS must be a multiple of threads per line");
  fft_passes<T, N, THREADS, 0>(buf, nlines, ls, tw);
  // results are read by other warps afterwards
  __syncthreads();
}

// Pass 0 of the plan with operands that the caller supplies from registers:
// s = begin(l) describes line l, fetch(s, i) loads its element i (typically
// a predicated global load) and fix(s, i, raw) turns the raw value into the
// operand (shift, mask, derivative ...).  A thread issues the fetches of all
// its operands before the first fix, so that its loads are in flight
// together whatever branches fix takes.  Pass 0 has no twiddles; its output
// goes to the line in shared memory, so the staging copy of the input (a
// shared-memory write and read per element) disappears.
template <typename T, int N, int THREADS, typename Begin, typename Fetch, typename Fix>
__device__ __forceinline__ void fft_pass0_load(C2<T>* buf, int nlines, int ls, Begin begin, Fetch fetch, Fix fix) {
  using C = C2<T>;
  using PL = FFTPlan<T, N>;
  constexpr int R = PL::rad(0), E = PL::E, P = PL::P;
  constexpr int LPR = THREADS / P;
  constexpr int NB = E / R;
  const int lr = threadIdx.x / P, t = threadIdx.x % P;
  for (int l0 = 0; l0 < nlines; l0 += LPR) {
    const int l = l0 + lr;
    if (l < nlines) {
      const auto s = begin(l);
      C v[E];
#pragma unroll
      for (int q = 0; q < NB; q++)
#pragma unroll
        for (int r = 0; r < R; r++) v[q * R + r] = fetch(s, t + q * P + r * (N / R));
#pragma unroll
      for (int q = 0; q < NB; q++)
#pragma unroll
        for (int r = 0; r < R; r++) v[q * R + r] = fix(s, t + q * P + r * (N / R), v[q * R + r]);
      C* line = buf + (size_t)l * ls;
#pragma unroll
      for (int q = 0; q < NB; q++) {
        const int j = t + q * P;
        dft_s<R, 1>(v + q * R);
#pragma unroll
        for (int r = 0; r < R; r++) line[pad32(j * R + r)] = v[q * R + r];
      }
    }
  }
}

// fft_lines with pass 0 fed by fft_pass0_load; waits for the caller's
// cp.async twiddle copies before the passes that use them.
template <typename T, int N, int THREADS, typename Begin, typename Fetch, typename Fix>
__device__ __forceinline__ void fft_lines_load(C2<T>* buf, int nlines, int ls, const C2<T>* tw, Begin begin,
                                               Fetch fetch, Fix fix) {
  static_assert(THREADS % FFTPlan<T, N>::P == 0, "THREADS must be a multiple of threads per line");
  fft_pass0_load<T, N, THREADS>(buf, nlines, ls, begin, fetch, fix);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  fft_passes<T, N, THREADS, 1>(buf, nlines, ls, tw);
  __syncthreads();
}

// The last pass of the plan with its outputs handed to the caller:
// store(s, base, vals, R, NS) with s = begin(l) receives elements base +
// r NS (r < R, natural order) of line l in vals[r] (R and NS as
// std::integral_constant), typically as global stores, so the pass output is
// not written to shared memory and read back.
template <typename T, int N, int THREADS, typename Begin, typename Store>
__device__ __forceinline__ void fft_pass_last_store(const C2<T>* buf, int nlines, int ls, const C2<T>* tw,
                                                    Begin begin, Store store) {
  using C = C2<T>;
  using PL = FFTPlan<T, N>;
  constexpr int PASS = PL::NPASS - 1;
  constexpr int R = PL::rad(PASS), NS = PL::ns(PASS), E = PL::E, P = PL::P;
  constexpr int LPR = THREADS / P, NB = E / R;
  const int lr = threadIdx.x / P, t = threadIdx.x % P;
  for (int l0 = 0; l0 < nlines; l0 += LPR) {
    const int l = l0 + lr;
    if (l < nlines) {
      C v[E];
      pass_butterflies<C, N, R, NS, E, P, PL::fact(PASS)>(buf + (size_t)l * ls, t, tw + PL::twoff(PASS), v);
      const auto s = begin(l);
#pragma unroll
      for (int q = 0; q < NB; q++) {
        const int j = t + q * P;
        const int k = j % NS;
        store(s, (j / NS) * NS * R + k, v + q * R, std::integral_constant<int, R>(),
              std::integral_constant<int, NS>());
      }
    }
  }
}

template <typename T, int N, int THREADS, int PASS, int LAST>
__device__ __forceinline__ void fft_passes_until(C2<T>* buf, int nlines, int ls, const C2<T>* tw) {
  using PL = FFTPlan<T, N>;
  if constexpr (PASS < LAST) {
    constexpr int R = PL::rad(PASS);
    constexpr int NS = PL::ns(PASS);
    fft_pass<C2<T>, N, R, NS, PL::E, PL::P, THREADS, PL::fact(PASS)>(buf, nlines, ls, tw + PL::twoff(PASS));
    fft_passes_until<T, N, THREADS, PASS + 1, LAST>(buf, nlines, ls, tw);
  }
}

// Whole transform with pass 0 fed by fetch and fix (fft_pass0_load) and the last pass
// handing its outputs to store: shared memory holds only the exchanges
// between passes.  Needs a plan of two passes or more.
template <typename T, int N, int THREADS, typename LBegin, typename Fetch, typename Fix, typename SBegin,
          typename Store>
__device__ __forceinline__ void fft_lines_load_store(C2<T>* buf, int nlines, int ls, const C2<T>* tw,
                                                     LBegin lbegin, Fetch fetch, Fix fix, SBegin sbegin,
                                                     Store store) {
  using PL = FFTPlan<T, N>;
  static_assert(PL::NPASS >= 2, "load and store passes must differ");
  static_assert(THREADS % PL::P == 0, "THREADS must be a multiple of threads per line");
  fft_pass0_load<T, N, THREADS>(buf, nlines, ls, lbegin, fetch, fix);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  fft_passes_until<T, N, THREADS, 1, PL::NPASS - 1>(buf, nlines, ls, tw);
  fft_pass_last_store<T, N, THREADS>(buf, nlines, ls, tw, sbegin, store);
}

// Host: build the twiddle table of FFTPlan<T,N> (pass p >= 1 table is
// [r][k] = W_N^(r k N/(Ns R)), r < R, k < Ns; factored passes hold the rows
// r0 = 0..7 and 8 r1, r1 = 0..R/8-1, see plan_fact).
template <typename T, int N>
void build_twiddles(C2<T>* out) {
  using PL = FFTPlan<T, N>;
  auto w = [](long m) {
    // accurate angle: reduce m/N to [0,1) exactly in integers
    m %= N;
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)N;
    return cmk<C2<T>>((T)cosl(ang), (T)sinl(ang));
  };
  for (int p = 1; p < PL::NPASS; p++) {
    const int R = PL::rad(p), NS = PL::ns(p), off = PL::twoff(p);
    const long s = N / (NS * R);
    if (PL::fact(p)) {
      for (int k = 0; k < NS; k++) {
        for (int r0 = 0; r0 < 8; r0++) out[off + r0 * NS + k] = w((long)r0 * k * s);
        for (int r1 = 0; r1 < R / 8; r1++) out[off + (8 + r1) * NS + k] = w((long)8 * r1 * k * s);
      }
    } else {
      for (int r = 0; r < R; r++)
        for (int k = 0; k < NS; k++) out[off + r * NS + k] = w((long)r * k * s);
    }
  }
}

}  // namespace psdns
