// stage_kernels.cuh -- the five fused kernels of one RK stage.
//
// Device data layout (one box, n^3, kxn kx columns, xz_tot cylinder columns):
//   u, un  [v][a][y]                 y-cylinders, the reference's uy(ny,num_al,v)
//   ub     [v][a/TB][y][a%TB]         cylinder data with y and a swapped in
//                                    blocks of TB columns (TB_I inverse, TB_F forward)
//   uz     [v][y][z/TZ][x][z%TZ]      z-pencils for x < kxn, blocked in z so that an
//                                    x-line tile of TZ lines is one contiguous block
// Per stage:
//   K1 k_yinv   : phase shift + mask (phshift.f:71-135), y backward FFT
//                 (kxcomm1_clean.f:118), transposed store into ub
//   K2 k_zinv   : cylinder unpack with zero fill (kxcomm1_clean.f:205-255),
//                 z backward FFT (itransform_vel.f:80-94), store into uz
//   K3 k_xchain : x complex-to-real (kxcomm2.f:308-321), the five products and
//                 velmax (realspace_vel.f:105-114), x real-to-complex times 1/n
//                 (xkcomm1.f:97,135); the physical field never leaves the chip
//   K4 k_zfwd   : z forward FFT (transform.f:129-138), derivative combination
//                 (transform.f:230-234), cylinder pack (xkcomm2.f:96-125) into ub
//   K5 k_yfwd   : y forward FFT (xkcomm2.f:229), wavespace closure
//                 (wavespace_vel.f:163-174), proc4a/proc4b update, projection and
//                 Eswaran-Pope forcing (proc4a.f:418-651, proc4b.f:38-205)
#pragma once
#include <type_traits>

#include "fft_core.cuh"
#include "tc_dft.cuh"

namespace psdns {

struct Geo {
  int n, kxn, xz_tot, nzt, nab_i, nab_f;
  const int* colstart;   // [kxn+1]
  const int* ax;         // [xz_tot] x index of column a
  const int* az;         // [xz_tot] z index (0..n-1) of column a
  const int* kymax;      // [xz_tot] largest |ky| inside the sphere
  // a batch of boxes of the same n (ensembles): box b's u/un, ub and uz start
  // b * sbox, b * bbox, b * zbox elements after box 0's (0 for one box)
  size_t sbox = 0, bbox = 0, zbox = 0;
};

// kx columns kept for a box of n: kxn = min(n/2, floor(kmax) + 1) with kmax
// = sqrt(2) n / 3 (init.f:29); floor(sqrt(2) n / 3) is the largest m with
// 9 m^2 <= 2 n^2.  A compile-time constant of the kernels' template n.
__host__ __device__ constexpr int kxn_of(int n) {
  int m = 0;
  while (9LL * (m + 1) * (m + 1) <= 2LL * n * n) m++;
  return m + 1 < n / 2 ? m + 1 : n / 2;
}

template <typename T> struct StageTables {
  const C2<T>* sx;   // [n/2+1] shift factors of this stage
  const C2<T>* sy;   // [n]
  const C2<T>* sz;   // [n]
  const T* xfac;     // [n/2+1] integrating factors
  const T* yfac;     // [n]
  const T* zfac;     // [n]
  const T* xdif;     // [n/2+1] scalar factors xfac^(1/Sc) (step.f:387-407)
  const T* ydif;     // [n]
  const T* zdif;     // [n]
  const C2<T>* forc; // for(kfor,k2fo,k2fo,3) or null
  int kfor, k2fo;
  double kforce2;    // kforce^2
  T b11, b22, b33;
  T norm;            // dt2/ny/nz
  const T* spf;      // spline prefilter 6/(4+2cos(2 pi k/n)): [n/2+1] x, [n] y, [n] z
  // batches: box b's tables start tbox bytes after box (b-1)'s, and its
  // norm is normv[b] (normv null: one box, norm above)
  size_t tbox = 0;
  const T* normv = nullptr;
  double tdk = 1.0;  // shell width of the transfer spectrum, min(beta) (trfsp.f:43)

  __device__ __forceinline__ StageTables at_box(int b) const {
    StageTables t = *this;
    if (tbox != 0) {
      const size_t o = (size_t)b * tbox;
      auto sh = [o](auto* p) { return p ? (decltype(p))((const char*)p + o) : p; };
      t.sx = sh(sx); t.sy = sh(sy); t.sz = sh(sz);
      t.xfac = sh(xfac); t.yfac = sh(yfac); t.zfac = sh(zfac);
      t.xdif = sh(xdif); t.ydif = sh(ydif); t.zdif = sh(zdif);
    }
    if (normv) t.norm = normv[b];
    return t;
  }
};

// per-precision tile sizes: TB_I = columns per K1 block (64 B runs in ub
// for K2), TB_F = columns per K5 block, TZ = z lines per K3 tile (32 B
// runs), XT2 = x lines per K2 block (K4's: k4_xt), YT4 = y rows per K4 block.
// Eight lines per block keep two to three blocks resident per SM, so that
// one block's copies overlap another's transforms; sixteen-line blocks (one
// per SM) measured slower for K1 and K4.  The z transforms run smaller
// blocks in FP32: K2 four lines (XT2 = 4) and K4 four (two x lines of two
// fields), 4-9% faster at 512^3 and 1024^3 than eight and eight; sixteen-line
// K2 blocks were 30% slower.
// The inverse ub layout is blocked by TBL_I = 2 TB_I columns (128 B runs for
// K2's reads), filled by pairs of K1 blocks.
template <typename T> struct Tiles;
template <> struct Tiles<float> {
  static constexpr int TB_I = 8, TBL_I = 16, TB_F = 4, TBL_F = 8, TZ = 4, XT2 = 4, YT4 = 1;
};
template <> struct Tiles<double> {
  static constexpr int TB_I = 4, TBL_I = 8, TB_F = 2, TBL_F = 4, TZ = 2, XT2 = 4, YT4 = 1;
};

// x lines per K4 block by box size (dbl: FP64 state).  FP32: four from
// 512^3 up (1024^3: 11.44 ms against 11.77 with two), two below (256^3:
// 0.148 ms against 0.150)
__host__ __device__ constexpr int k4_xt(bool dbl, int n) { return dbl ? 2 : (n >= 512 ? 4 : 2); }

// elements of one variable of the forward ub layout [a/TBL_F][y][a%TBL_F]
// (K4 writes 64-byte runs; K5 blocks of TB_F columns read halves)
template <typename T>
__host__ __device__ __forceinline__ size_t ubf_var_elems(int nab_f, int n) {
  constexpr int R = Tiles<T>::TBL_F / Tiles<T>::TB_F;
  return (size_t)((nab_f + R - 1) / R * R) * Tiles<T>::TB_F * n;
}

// elements of one variable of the inverse ub layout [a/TBL_I][y][a%TBL_I]
template <typename T>
__host__ __device__ __forceinline__ size_t ubi_var_elems(int nab_i, int n) {
  constexpr int R = Tiles<T>::TBL_I / Tiles<T>::TB_I;
  return (size_t)((nab_i + R - 1) / R * R) * Tiles<T>::TB_I * n;
}

template <int N> __device__ __forceinline__ int kwave(int i) { return i > N / 2 ? i - N : i; }

__device__ __forceinline__ bool mask_ok(const Geo& g, int a, int y, int n) {
  if (y == n / 2) return false;
  int ky = y > n / 2 ? n - y : y;
  return ky <= __ldg(g.kymax + a);
}

// Asynchronous global -> shared copies of one complex element (cp.async,
// 8 or 16 bytes).  A thread issues all of its copies before waiting, so a
// block keeps its whole tile in flight; after cp_async_wait_all() the
// thread's own copies have landed (other threads' copies need a barrier).
template <typename C>
__device__ __forceinline__ void cp_async_elem(C* smem_dst, const C* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  if constexpr (sizeof(C) == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
  }
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// twiddles are copied asynchronously: every kernel calls cp_async_wait_all()
// and __syncthreads() before its first FFT
template <typename T, int N>
__device__ __forceinline__ void load_twiddles(C2<T>* tw_s, const C2<T>* __restrict__ tw_g) {
  constexpr int TS = FFTPlan<T, N>::TWSIZE;
  for (int i = threadIdx.x; i < TS; i += blockDim.x) cp_async_elem(tw_s + i, tw_g + i);
}

// threads of a block that transforms LINES lines at once (capped at CAP, at
// least one warp, and a multiple of the P threads of a line: P = 6 at
// n = 48)
__host__ __device__ constexpr int round_up(int a, int m) { return (a + m - 1) / m * m; }
__host__ __device__ constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }
template <typename T, int N, int LINES, int CAP = 256>
struct Launch {
  static constexpr int P = FFTPlan<T, N>::P;
  static constexpr int want = LINES * P;
  static constexpr int THREADS = round_up((want >= CAP ? CAP : (want < 32 ? 32 : want)), P);
  static_assert(THREADS % P == 0, "threads per line must divide the block");
};

template <int N> struct LS { static constexpr int value = N + N / 32 + 4; };

// K1 and K4: one warp per line at n = 1024 FP32
template <typename T, int N>
struct K1Launch : Launch<T, N, Tiles<T>::TB_I, 1024> {};
// K4 with XT x lines per block: three fields of every x line at once
// (register-fed form, phase 1 of k_zfwd), or two (tensor-core form)
template <typename T, int N, int XT, bool TCM = false>
struct K4LaunchX : Launch<T, N, (TCM ? 2 : 3) * XT * Tiles<T>::YT4, 1024> {
  static constexpr int NF = TCM ? 2 : 3;
  // resident blocks the registers are sized for: about 112 registers a
  // thread in the register-fed form (its last pass holds a line's operands
  // and the store addresses), one to eight blocks
  static constexpr int TH = Launch<T, N, NF * XT * Tiles<T>::YT4, 1024>::THREADS;
  static constexpr int MINB_F = 65536 / (TH * 112) < 1 ? 1 : (65536 / (TH * 112) > 8 ? 8 : 65536 / (TH * 112));
  static constexpr int MINB = TCM ? 2 : MINB_F;
  static constexpr size_t SMEM =
      sizeof(C2<T>) * (FFTPlan<T, N>::TWSIZE + (size_t)NF * XT * Tiles<T>::YT4 * LS<N>::value);
};
template <typename T, int N>
struct K4Launch : K4LaunchX<T, N, k4_xt(sizeof(T) == 8, N)> {};

// K5 holds one CTA per SM (its (4 + nc) * TB_F lines fill shared memory), so
// it runs every line of a block at once
template <typename T, int N, int NC>
struct K5Launch : Launch<T, N, (4 + NC) * Tiles<T>::TB_F, 1024> {};

// Mixed-precision form of the stage kernels (template flag TCM, FP32 state
// at n = 1024): every 1024-point transform runs on the tensor cores
// (tc_dft.cuh, split-BF16 operands, FP32 accumulation) instead of the FP32
// Stockham passes.  TcArgs: the B operands and twiddles of tc_dft.cuh and
// the error word its bounded waits report to.  The shared-memory tail (B
// operands, barrier, TMEM address) follows the kernel's own lines.
struct TcArgs {
  const uint4* btab = nullptr;
  const float2* tw2 = nullptr;
  unsigned* err = nullptr;
};
constexpr size_t kTcTail = tc::kBBytes + 16;
// z tiles of the tensor-core kernels, independent of Tiles<float>: an operand
// tile (32 KB) overlays four lines, so every line buffer that one transform
// call runs on holds at least four lines
constexpr int kTcXT2 = 8, kTcXT4 = 4;
// TMEM columns for nlines lines: 64 per tile of four, as a power of two
__host__ __device__ constexpr int tc_cols(int nlines) {
  int c = 64 * ((nlines + 3) / 4), p = 32;
  while (p < c) p *= 2;
  return p;
}
template <int NCOLS>
__device__ __forceinline__ void tc_begin(tc::Work& w, unsigned char* tail, const TcArgs& a) {
  tc::setup<NCOLS>(w, tail, reinterpret_cast<uint64_t*>(tail + tc::kBBytes),
                   reinterpret_cast<uint32_t*>(tail + tc::kBBytes + 8), a.btab, a.tw2, a.err);
}
// in-place forward transform of lines in shared memory, FP32 or tensor cores
template <typename T, int N, int THREADS, bool TCM>
__device__ __forceinline__ void lines_fft(C2<T>* buf, int nlines, int ls, const C2<T>* tw, tc::Work& w) {
  if constexpr (TCM)
    tc::fft1024_lines<THREADS>(buf, nlines, ls, w);
  else
    fft_lines<T, N, THREADS>(buf, nlines, ls, tw);
}

// ---------------------------------------------------------------------------
// K1: phase shift + mask + y backward FFT, transposed store to ub (TB_I block)
// grid (ceil(xz_tot/TB_I), 3); one block = one ub block of TB_I columns
// ---------------------------------------------------------------------------
template <typename T, int N, bool SPL = false, int NC = 0, bool TCM = false>
__global__ void __launch_bounds__(K1Launch<T, N>::THREADS, TCM ? 2 : 3)
k_yinv(Geo g, StageTables<T> st_all, const C2<T>* __restrict__ u, C2<T>* __restrict__ ub,
       const C2<T>* __restrict__ tw_g, TcArgs tca = TcArgs()) {
  // grid (nab_i, 3 + 2 nc, boxes)
  const int box = blockIdx.z;
  const StageTables<T> st = st_all.at_box(box);
  u += box * g.sbox;
  ub += box * g.bbox;
  // NC = 1 (one passive scalar, grid.y = 5): ub variable 3 is the shifted
  // scalar and variable 4 its y gradient i b22 ky theta (phase1.f:52-64)
  // SPL: also divide by the cubic B-spline symbol, (4 + 2 cos(2 pi k/n))/6 per
  // axis, so that the backward transform yields the periodic spline
  // coefficients of the shifted-grid field (the circulant tridiagonal systems
  // that splx.f/splz_m.f/sply.f solve in physical space)
  using C = C2<T>;
  constexpr int TB = Tiles<T>::TB_I;
  constexpr int THREADS = K1Launch<T, N>::THREADS;
  constexpr int L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* buf = tw + FFTPlan<T, N>::TWSIZE;
  load_twiddles<T, N>(tw, tw_g);
  const int at = blockIdx.x, v = blockIdx.y;
  const int src = v < 3 ? v : 3;
  const int a0 = at * TB;
  const size_t vs = (size_t)g.xz_tot * N;
  // the TB columns are contiguous in u; pass 0 of the transform loads its
  // operands straight from them, shifted (and masked, differentiated,
  // prefiltered) in registers; masked entries are not read
  const C* colbase = u + src * vs + (size_t)a0 * N;
  struct Col { const C* col; C sxz; T fx, fz; int kym; };
  auto begin = [&](int l) {
    Col s{colbase + (size_t)l * N, cmk<C>(0, 0), T(0), T(0), -1};
    const int a = a0 + l;
    if (a < g.xz_tot) {
      const int x = __ldg(g.ax + a), z = __ldg(g.az + a);
      s.sxz = cmul(__ldg(st.sx + x), __ldg(st.sz + z));
      s.kym = __ldg(g.kymax + a);
      if constexpr (SPL) { s.fx = __ldg(st.spf + x); s.fz = __ldg(st.spf + (N / 2 + 1) + N + z); }
    }
    return s;
  };
  // fetch: the shifted entry (zero where masked); fix: derivative, prefilter
  // and the conjugation of the backward transform (zero stays zero)
  auto fetch = [&](const Col& s, int y) {
    const int ky = y > N / 2 ? N - y : y;
    C val = cmk<C>(0, 0);
    if (y != N / 2 && ky <= s.kym) {
      const C sh = cmul(__ldg(st.sy + y), s.sxz);
      val = cmul(__ldg(s.col + y), sh);
    }
    return val;
  };
  auto fix = [&](const Col& s, int y, C val) {
    if constexpr (NC > 0) {
      if (v == 4) {
        const T bk = st.b22 * T(kwave<N>(y));
        val = cmk<C>(-bk * val.y, bk * val.x);
      }
    }
    if constexpr (SPL) val = cscale(s.fx * __ldg(st.spf + (N / 2 + 1) + y) * s.fz, val);
    return cconj(val);
  };
  if constexpr (TCM) {
    tc::Work w;
    constexpr int NCOL = tc_cols(TB);
    tc_begin<NCOL>(w, reinterpret_cast<unsigned char*>(buf + TB * L), tca);
    auto line = [&](int l) { return buf + (size_t)l * L; };
    tc::fft1024<THREADS>(
        TB, w, reinterpret_cast<unsigned char*>(buf), (uint32_t)(4 * L * sizeof(C)), begin,
        [&](const Col& s, int y) { return fix(s, y, fetch(s, y)); }, line,
        [](C* p, int k, C v) { p[pad32(k)] = v; });
    tc::teardown<NCOL>(w);
  } else {
    fft_lines_load<T, N, THREADS>(buf, TB, L, tw, begin, fetch, fix);
  }
  // columns a0 + l sit at ((a / TBL) n + y) TBL + a % TBL of variable v: a
  // block writes 64-byte halves of the 128-byte runs (a sequential pair of
  // groups per block measured slower than independent blocks)
  constexpr int TBL = Tiles<T>::TBL_I, R = TBL / TB;
  C* out = ub + (size_t)v * ubi_var_elems<T>(g.nab_i, N) + (size_t)(at / R) * N * TBL + (at % R) * TB;
  for (int e = threadIdx.x; e < TB * N; e += THREADS) {
    const int y = e / TB, l = e % TB;
    out[y * TBL + l] = cconj(buf[l * L + pad32(y)]);
  }
}

// K1 grid.x: one block per TB_I columns
template <typename T>
__host__ __device__ __forceinline__ int k1_blocks(int nab_i) { return nab_i; }

// ---------------------------------------------------------------------------
// K2: cylinder unpack (zero fill) + z backward FFT, store to uz
// grid (n, ceil(kxn/XT2), 3)
// ---------------------------------------------------------------------------
// XTO > 0: XTO x lines per block instead of Tiles<T>::XT2 (a tile variant
// of the ensemble autotuner; every line is transformed the same way)
// The FP32 velocity form's registers are sized for five resident blocks
// (102 a thread at 128 threads): 1024^3 5.65 -> 5.33 ms against three; six
// blocks (85, small spills) 6.01 ms.
template <typename T, int N, int NC = 0, bool GRAD = false, bool TCM = false, int XTO = 0>
__global__ void __launch_bounds__(Launch<T, N, (XTO > 0 ? XTO : Tiles<T>::XT2)>::THREADS,
                                  TCM ? 2 : (sizeof(T) == 4 && NC == 0 && !GRAD ? 5 : 3))
k_zinv(Geo g, const C2<T>* __restrict__ ub, C2<T>* __restrict__ uz, const C2<T>* __restrict__ tw_g, T b11 = T(1),
       T b33 = T(1), TcArgs tca = TcArgs()) {
  // GRAD (grid.z = 2): uz slot 0 = i b11 kx u, slot 1 = i b33 kz w, the
  // gradients whose moments vgmomt.f takes (itransform.f:222-230)
  // NC = 1 (grid.z = 6): uz slot 3 = y gradient of the scalar (ub 4), slot
  // 4 = i b11 kx theta and slot 5 = i b33 kz theta (both from ub 3),
  // itransform.f:188-198
  using C = C2<T>;
  constexpr int XT = XTO > 0 ? XTO : Tiles<T>::XT2, TZ = Tiles<T>::TZ;
  static_assert(!TCM || XT >= 4, "an operand tile overlays four lines");
  constexpr int THREADS = Launch<T, N, XT>::THREADS;
  constexpr int L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* buf = tw + FFTPlan<T, N>::TWSIZE;
  load_twiddles<T, N>(tw, tw_g);
  // grid (n, ceil(kxn / XT2), (3 + 3 nc) * boxes)
  constexpr int NVZ = GRAD ? 2 : 3 + 3 * NC;
  const int y = blockIdx.x, x0 = blockIdx.y * XT, v = blockIdx.z % NVZ, box = blockIdx.z / NVZ;
  ub += box * g.bbox;
  uz += box * g.zbox;
  const int x1 = min(x0 + XT, g.kxn);
  const int nl = x1 - x0;
  const int sv = GRAD ? (v == 0 ? 0 : 2) : (v < 3 ? v : (v == 3 ? 4 : 3));
  constexpr int TBL = Tiles<T>::TBL_I;
  const C* src = ub + (size_t)sv * ubi_var_elems<T>(g.nab_i, N);
  // line l, entry z: column x0 + l holds kz = 0..kc then -kc..-1 (count
  // 2 kc + 1, mpisetup.f:322-357), so its cylinder index follows from
  // colstart alone; pass 0 of the transform reads the entries straight from
  // ub (consecutive z of a warp are consecutive columns), the cut band is zero
  struct Line { int ac, kc, x; };
  auto begin = [&](int l) {
    const int ac = __ldg(g.colstart + x0 + l);
    return Line{ac, (__ldg(g.colstart + x0 + l + 1) - ac - 1) / 2, x0 + l};
  };
  auto fetch = [&](const Line& s, int z) {
    if (z > s.kc && z < N - s.kc) return cmk<C>(0, 0);
    const int a = s.ac + (z <= s.kc ? z : z - N + 2 * s.kc + 1);
    return __ldg(src + ((size_t)((unsigned)a / TBL) * N + y) * TBL + ((unsigned)a % TBL));
  };
  auto fix = [&](const Line& s, int z, C val) {
    if constexpr (GRAD) {
      const T bk = v == 0 ? b11 * T(s.x) : b33 * T(kwave<N>(z));
      val = cmk<C>(-bk * val.y, bk * val.x);
    } else if constexpr (NC > 0) {
      if (v >= 4) {
        const T bk = v == 4 ? b11 * T(s.x) : b33 * T(kwave<N>(z));
        val = cmk<C>(-bk * val.y, bk * val.x);
      }
    }
    return cconj(val);
  };
  // the last pass stores its outputs straight to uz: line l, entry z at
  // ((v n + y) nzt + z / TZ) kxn + x0 + l) TZ + z % TZ (consecutive z of a
  // warp fill whole 32-byte sectors)
  const size_t vbase = ((size_t)v * N + y) * g.nzt;
  constexpr size_t zstride = (size_t)kxn_of(N) * TZ;   // g.kxn, as a constant
  auto sbegin = [&](int l) { return uz + (vbase * g.kxn + x0 + l) * TZ; };
  auto store = [&](C* d, int base, const C* vals, auto Rc, auto NSc) {
    constexpr int R = decltype(Rc)::value, NS = decltype(NSc)::value;
    static_assert(NS % TZ == 0, "last-pass stride must keep z % TZ");
    C* p = d + ((unsigned)base / TZ) * zstride + (unsigned)base % TZ;
#pragma unroll
    for (int r = 0; r < R; r++) p[(size_t)(r * (NS / TZ)) * zstride] = cconj(vals[r]);
  };
  if constexpr (TCM) {
    tc::Work w;
    constexpr int NCOL = tc_cols(XT);
    tc_begin<NCOL>(w, reinterpret_cast<unsigned char*>(buf + XT * L), tca);
    tc::fft1024<THREADS>(
        nl, w, reinterpret_cast<unsigned char*>(buf), (uint32_t)(4 * L * sizeof(C)), begin,
        [&](const Line& s, int z) { return fix(s, z, fetch(s, z)); }, sbegin,
        [&](C* d, int z, C v) { d[((unsigned)z / TZ) * zstride + (unsigned)z % TZ] = cconj(v); });
    tc::teardown<NCOL>(w);
  } else {
    fft_lines_load_store<T, N, THREADS>(buf, nl, L, tw, begin, fetch, fix, sbegin, store);
  }
}

// ---------------------------------------------------------------------------
// K3: x-line chain.  grid (nzt, n): one block = TZ x-lines (z = zt*TZ + zz)
// at one y.  Two real lines are carried in one complex FFT (pairs zz=2p,2p+1).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void atomic_max_pos(unsigned long long* addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

template <typename T, int N>
__device__ __forceinline__ void xchain_store(const Geo& g, const C2<T>* buf, int nbuf, int L,
                                             C2<T>* __restrict__ uz, int slot0, int y, int zt,
                                             T half_factor) {
  using C = C2<T>;
  constexpr int TZ = Tiles<T>::TZ, NPAIR = TZ / 2;
  const int kxn = g.kxn;
  // thread -> fixed pair p, x strided by blockDim/NPAIR (no runtime division)
  const int p = threadIdx.x % NPAIR, x0 = threadIdx.x / NPAIR, xs = blockDim.x / NPAIR;
  for (int b = 0; b < nbuf; b++)
  for (int x = x0; x < kxn; x += xs) {
    const C* line = buf + (b * NPAIR + p) * L;
    const C Y = line[pad32(x)];
    const C Yn = line[pad32(x == 0 ? 0 : N - x)];
    const C A = cmk<C>((Y.x + Yn.x) * half_factor, (Y.y - Yn.y) * half_factor);
    const C B = cmk<C>((Y.y + Yn.y) * half_factor, (Yn.x - Y.x) * half_factor);
    C* dst = uz + ((((size_t)(slot0 + b) * N + y) * g.nzt + zt) * kxn + x) * TZ + 2 * p;
    dst[0] = A;
    dst[1] = B;
  }
}

// Load NV x-line tiles (uz slots v0..v0+NV-1, TZ lines each) and pack two
// real lines per complex line: Z(k) = A(k) + i B(k), with the Hermitian
// extension and the imaginary part of the kx=0 term dropped; stored
// conjugated (backward transform by conjugation).  All loads of a thread are
// issued before the first shared-memory store.
template <typename T, int N, int NV, int THREADS>
__device__ __forceinline__ void xchain_pack(const Geo& g, const C2<T>* __restrict__ uz, int v0, int y, int zt,
                                            C2<T>* bufU, int L) {
  using C = C2<T>;
  constexpr int TZ = Tiles<T>::TZ, NPAIR = TZ / 2;
  constexpr int XST = THREADS / NPAIR;
  constexpr int XI = (N / 2 + XST - 1) / XST;
  const int kxn = g.kxn;
  const int p = threadIdx.x % NPAIR, xth = threadIdx.x / NPAIR;
  C A[NV][XI], B[NV][XI];
#pragma unroll
  for (int v = 0; v < NV; v++)
#pragma unroll
    for (int i = 0; i < XI; i++) {
      const int x = xth + i * XST;
      if (x < kxn) {
        const C* src = uz + ((((size_t)(v0 + v) * N + y) * g.nzt + zt) * kxn + x) * TZ + 2 * p;
        if constexpr (sizeof(C) == 8) {
          const float4 q = *reinterpret_cast<const float4*>(src);
          A[v][i] = cmk<C>(q.x, q.y);
          B[v][i] = cmk<C>(q.z, q.w);
        } else {
          A[v][i] = src[0];
          B[v][i] = src[1];
        }
      }
    }
#pragma unroll
  for (int v = 0; v < NV; v++)
#pragma unroll
    for (int i = 0; i < XI; i++) {
      const int x = xth + i * XST;
      if (x < kxn) {
        const C a = A[v][i], b = B[v][i];
        C* line = bufU + (v * NPAIR + p) * L;
        if (x == 0) {
          line[pad32(0)] = cmk<C>(a.x, -b.x);
        } else {
          line[pad32(x)] = cmk<C>(a.x - b.y, -(a.y + b.x));
          line[pad32(N - x)] = cmk<C>(a.x + b.y, -(b.x - a.y));
        }
      }
    }
}

// Register-level pair packing for plans of two passes whose last radix is
// the operand count E (so P = R0 threads per line, inside one warp).  Thread
// t of a line then holds the elements t + P m (m < R1) both as the operands
// of pass 0 and as the outputs of the last pass, and the Hermitian partner
// N - x of its element x sits in lane P - t (slot R1 - 1 - m; lane 0 pairs
// with itself, slot R1 - m).  The packing before the inverse transform and
// the unpacking after the forward one then exchange values by warp shuffles
// instead of a shared-memory round trip of every line.
template <typename T, int N>
struct XFuse {
  using PL = FFTPlan<T, N>;
  static constexpr bool value =
      is_pow2(N) && PL::NPASS == 2 && PL::rad(1) == PL::E && PL::P <= 32 && (32 % PL::P) == 0;
};

// xchain_pack followed by pass 0 of the transform, with the operands
// loaded from uz into registers: line l = v NPAIR + p gets
// conj(A + i B) of the real lines z = zt TZ + 2p, 2p + 1 of slot v0 + v (the
// band kx in [kxn, N - kxn] zero), and pass 0's output goes to shared memory.
// Every thread of the block runs the same rounds (the shuffles name whole
// warps); loads and stores are predicated on the line being one of NV NPAIR.
template <typename T, int N, int NV, int THREADS>
__device__ __forceinline__ void xchain_load_pass0(const Geo& g, const C2<T>* __restrict__ uz, int v0, int y,
                                                  int zt, C2<T>* buf, int L) {
  using C = C2<T>;
  using PL = FFTPlan<T, N>;
  static_assert(XFuse<T, N>::value, "plan without register-level packing");
  constexpr int TZ = Tiles<T>::TZ, NPAIR = TZ / 2;
  constexpr int R0 = PL::rad(0), R1 = PL::rad(1), P = PL::P, E = PL::E, H = R1 / 2;
  constexpr int LPR = THREADS / P, NB = E / R0;
  static_assert(THREADS % 32 == 0, "whole warps");
  const int kxn = g.kxn;
  const int lr = threadIdx.x / P, t = threadIdx.x % P;
  const int src = (P - t) & (P - 1);
  for (int l0 = 0; l0 < NV * NPAIR; l0 += LPR) {
    const int l = l0 + lr;
    const bool act = l < NV * NPAIR;
    const int v = act ? l / NPAIR : 0, p = l % NPAIR;
    const C* col = uz + (((size_t)(v0 + v) * N + y) * g.nzt + zt) * (size_t)kxn * TZ + 2 * p;
    C a[H], b[H];
#pragma unroll
    for (int m = 0; m < H; m++) {
      const int x = t + P * m;
      a[m] = cmk<C>(0, 0);
      b[m] = cmk<C>(0, 0);
      if (act && x < kxn) {
        if constexpr (sizeof(C) == 8) {
          const float4 q = *reinterpret_cast<const float4*>(col + (size_t)x * TZ);
          a[m] = cmk<C>(q.x, q.y);
          b[m] = cmk<C>(q.z, q.w);
        } else {
          a[m] = col[(size_t)x * TZ];
          b[m] = col[(size_t)x * TZ + 1];
        }
      }
    }
    // slot m < H: element x = t + P m; slot m >= H: element N - x' of lane
    // P - t's x' at slot R1 - 1 - m (lane 0: its own x' at slot R1 - m, and
    // zero at slot H, x = N/2)
    C z[R1];
#pragma unroll
    for (int m = H; m < R1; m++) z[m] = cmk<C>(0, 0);
#pragma unroll
    for (int m = 0; m < H; m++) {
      const C av = a[m], bv = b[m];
      z[m] = (t == 0 && m == 0) ? cmk<C>(av.x, -bv.x) : cmk<C>(av.x - bv.y, -(av.y + bv.x));
      const C mv = cmk<C>(av.x + bv.y, -(bv.x - av.y));   // element N - x
      const C got = cmk<C>(__shfl_sync(0xffffffffu, mv.x, src, P), __shfl_sync(0xffffffffu, mv.y, src, P));
      if (t != 0) {
        z[R1 - 1 - m] = got;
      } else if (m >= 1) {
        z[R1 - m] = mv;
      }
    }
    if (act) {
      C* line = buf + (size_t)l * L;
#pragma unroll
      for (int q = 0; q < NB; q++) {
        C w[R0];
#pragma unroll
        for (int r = 0; r < R0; r++) w[r] = z[q + NB * r];   // element t + q P + r R1
        dft_s<R0, 1>(w);
        const int j = t + q * P;
#pragma unroll
        for (int r = 0; r < R0; r++) line[pad32(j * R0 + r)] = w[r];
      }
    }
  }
}

// The last pass of the forward transform of nlines lines with xchain_store's
// unpacking done in registers: A(x), B(x) of the real lines z = zt TZ + 2p,
// 2p + 1 go to uz slot l / NPAIR for x < kxn.  Called by every thread of
// the block (whole warps per round).
template <typename T, int N, int THREADS>
__device__ __forceinline__ void xchain_last_store(const Geo& g, const C2<T>* buf, int nlines, int L,
                                                  const C2<T>* tw, C2<T>* __restrict__ uz, int y, int zt,
                                                  T half_factor) {
  using C = C2<T>;
  using PL = FFTPlan<T, N>;
  static_assert(XFuse<T, N>::value, "plan without register-level packing");
  constexpr int TZ = Tiles<T>::TZ, NPAIR = TZ / 2;
  constexpr int R1 = PL::rad(1), P = PL::P, E = PL::E, H = R1 / 2, NS = PL::ns(1);
  constexpr int LPR = THREADS / P;
  static_assert(NS == P && E == R1, "the last pass holds elements t + P m");
  const int kxn = g.kxn;
  const int lr = threadIdx.x / P, t = threadIdx.x % P;
  const int src = (P - t) & (P - 1);
  for (int l0 = 0; l0 < nlines; l0 += LPR) {
    const int l = l0 + lr;
    const bool act = l < nlines;
    C v[E];
    if (act) {
      pass_butterflies<C, N, R1, NS, E, P, PL::fact(1)>(buf + (size_t)l * L, t, tw + PL::twoff(1), v);
    } else {
#pragma unroll
      for (int m = 0; m < E; m++) v[m] = cmk<C>(0, 0);
    }
    const int b = act ? l / NPAIR : 0, p = l % NPAIR;
    C* col = uz + (((size_t)b * N + y) * g.nzt + zt) * (size_t)kxn * TZ + 2 * p;
#pragma unroll
    for (int m = 0; m < H; m++) {
      const int x = t + P * m;
      const C Y = v[m];
      const C sent = v[R1 - 1 - m];
      const C got = cmk<C>(__shfl_sync(0xffffffffu, sent.x, src, P), __shfl_sync(0xffffffffu, sent.y, src, P));
      const C Yn = t == 0 ? v[(R1 - m) % R1] : got;
      if (act && x < kxn) {
        const T ax = (Y.x + Yn.x) * half_factor, ay = (Y.y - Yn.y) * half_factor;
        const T bx = (Y.y + Yn.y) * half_factor, by = (Yn.x - Y.x) * half_factor;
        if constexpr (sizeof(C) == 8) {
          *reinterpret_cast<float4*>(col + (size_t)x * TZ) = make_float4(ax, ay, bx, by);
        } else {
          col[(size_t)x * TZ] = cmk<C>(ax, ay);
          col[(size_t)x * TZ + 1] = cmk<C>(bx, by);
        }
      }
    }
  }
}

// K3 runs the five output products of a tile as one batch of 5 * TZ/2
// lines: one warp per line at n = 1024 (a multiple of 32 threads, so that
// the velmax warp reduction sees whole warps)
template <typename T, int N, int NC>
struct K3Launch {
  static constexpr int P = FFTPlan<T, N>::P;
  static constexpr int NPAIR = Tiles<T>::TZ / 2;
  static constexpr int want = 5 * NPAIR * P;
  static constexpr int WP = 32 / gcd_c(32, P) * P;   // lcm(32, P): whole warps and whole lines
  static constexpr int THREADS = round_up(want, WP) > 1024 ? 1024 : round_up(want, WP);
  static_assert(THREADS % P == 0, "threads per line must divide the block");
  // twiddles + 5 product buffers (6 input buffers with a scalar) of TZ/2 lines
  static constexpr size_t SMEM =
      sizeof(C2<T>) * (FFTPlan<T, N>::TWSIZE + (size_t)(NC ? 6 : 5) * NPAIR * LS<N>::value);
  // tensor-core form: the line buffers rounded up to whole tiles of four
  // lines (the operands overlay them), then the tail
  static constexpr int LINES_TC = ((NC ? 6 : 5) * NPAIR + 3) / 4 * 4;
  static constexpr size_t SMEM_TC =
      sizeof(C2<T>) * (FFTPlan<T, N>::TWSIZE + (size_t)LINES_TC * LS<N>::value) + kTcTail;
};

template <typename T, int N, int NC = 0, bool TCM = false>
__global__ void __launch_bounds__(K3Launch<T, N, NC>::THREADS, TCM ? 1 : 2)
k_xchain(Geo g, C2<T>* __restrict__ uz, const C2<T>* __restrict__ tw_g, T b11, T b22, T b33,
         unsigned long long* velmax_bits, int want_velmax, T cb1 = T(0), T cb2 = T(0), T cb3 = T(0),
         TcArgs tca = TcArgs()) {
  // NC = 1: inputs also hold the scalar gradient (slots 3 = d/dy, 4 = d/dx,
  // 5 = d/dz); the advection term u.(G + grad theta) (itransform.f:522-530,
  // G = cb, init.f:42-45) is formed in physical space and goes to slot 5.
  using C = C2<T>;
  constexpr int TZ = Tiles<T>::TZ, NPAIR = TZ / 2;
  constexpr int NVIN = 3 + 3 * NC;
  constexpr int THREADS = K3Launch<T, N, NC>::THREADS;
  constexpr int L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* bufU = tw + FFTPlan<T, N>::TWSIZE;
  C* bufV = bufU + NPAIR * L;
  C* bufW = bufV + NPAIR * L;
  // with NC = 1, E and F hold the y and x gradients until the scalar term is done
  C* bufE = bufW + NPAIR * L;
  C* bufF = bufE + NPAIR * L;
  load_twiddles<T, N>(tw, tw_g);
  constexpr int NCOL = tc_cols(K3Launch<T, N, NC>::LINES_TC);
  tc::Work w;
  if constexpr (TCM)
    tc_begin<NCOL>(w, reinterpret_cast<unsigned char*>(bufU + K3Launch<T, N, NC>::LINES_TC * L), tca);
  // grid (nzt, n, boxes)
  const int zt = blockIdx.x, y = blockIdx.y, box = blockIdx.z;
  uz += box * g.zbox;
  velmax_bits += box;
  const int kxn = g.kxn;
  // the pair packing and unpacking in registers (XFuse) on the FFT path; the
  // tensor-core path and the other plans go through shared memory
  constexpr bool FUSE = !TCM && XFuse<T, N>::value;
  if constexpr (FUSE) {
    xchain_load_pass0<T, N, NVIN, THREADS>(g, uz, 0, y, zt, bufU, L);
    cp_async_wait_all();
    __syncthreads();
    fft_passes<T, N, THREADS, 1>(bufU, NVIN * NPAIR, L, tw);
    __syncthreads();
  } else {
    // zero the band kx in [kxn, n-kxn] (includes the Nyquist column)
    for (int e = threadIdx.x; e < NVIN * NPAIR * N; e += THREADS) {
      const int k = e % N;
      if (k >= kxn && k <= N - kxn) bufU[(e / N) * L + pad32(k)] = cmk<C>(0, 0);
    }
    xchain_pack<T, N, 3, THREADS>(g, uz, 0, y, zt, bufU, L);
    if constexpr (NC > 0) xchain_pack<T, N, 3, THREADS>(g, uz, 3, y, zt, bufU + 3 * NPAIR * L, L);
    cp_async_wait_all();
    __syncthreads();
    lines_fft<T, N, THREADS, TCM>(bufU, NVIN * NPAIR, L, tw, w);
  }
  // buffers now hold conj(a + i b): a = re, b = -im
  const T hf = T(0.5) / T(N);
  // realspace_vel.f:105-114, in place: slot 0 = b11 u^2 - bv2, 1 = uv,
  // 2 = b33 w^2 - bv2, 3 = vw (is1), 4 = uw (is2); velmax at stage 1.  With
  // a scalar, slot 5 = its advection term (buffer 5 held d/dz theta).
  double vm = 0.0;
  const double xn = (double)b11 * N, yn = (double)b22 * N, zn = (double)b33 * N;
  for (int e = threadIdx.x; e < NPAIR * N; e += THREADS) {
    const int i = (e / N) * L + pad32(e % N);
    const C U = bufU[i], V = bufV[i], W = bufW[i];
    if constexpr (NC > 0) {
      C* bufGZ = bufF + NPAIR * L;
      const C GY = bufE[i], GX = bufF[i], GZ = bufGZ[i];
      const T sa = U.x * (cb1 + GX.x) + V.x * (cb2 + GY.x) + W.x * (cb3 + GZ.x);
      const T sb = (-U.y) * (cb1 - GX.y) + (-V.y) * (cb2 - GY.y) + (-W.y) * (cb3 - GZ.y);
      bufGZ[i] = cmk<C>(sa, sb);
    }
    if (want_velmax) {
      double va = xn * fabs((double)U.x) + yn * fabs((double)V.x) + zn * fabs((double)W.x);
      double vb = xn * fabs((double)U.y) + yn * fabs((double)V.y) + zn * fabs((double)W.y);
      vm = fmax(vm, fmax(va, vb));
    }
    // the sign of b cancels in the mixed products
    bufF[i] = cmk<C>(U.x * W.x, U.y * W.y);
    bufE[i] = cmk<C>(V.x * W.x, V.y * W.y);
    const T ua = U.x, ub = -U.y, va = V.x, vb = -V.y, wa = W.x, wb = -W.y;
    const T bva = b22 * va * va, bvb = b22 * vb * vb;
    bufW[i] = cmk<C>(b33 * wa * wa - bva, b33 * wb * wb - bvb);
    bufV[i] = cmk<C>(ua * va, ub * vb);
    bufU[i] = cmk<C>(b11 * ua * ua - bva, b11 * ub * ub - bvb);
  }
  if (want_velmax) {
    // block max through warp shuffles then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
    if ((threadIdx.x & 31) == 0) atomic_max_pos<T>(velmax_bits, vm);
  }
  __syncthreads();
  if constexpr (FUSE) {
    // pass 0 in shared memory; each line's last pass runs on the warp that
    // wrote it, so a warp barrier (inside fft_pass) orders the two
    fft_passes_until<T, N, THREADS, 0, 1>(bufU, (5 + NC) * NPAIR, L, tw);
    xchain_last_store<T, N, THREADS>(g, bufU, (5 + NC) * NPAIR, L, tw, uz, y, zt, hf);
  } else {
    lines_fft<T, N, THREADS, TCM>(bufU, (5 + NC) * NPAIR, L, tw, w);
    if constexpr (TCM) tc::teardown<NCOL>(w);
    xchain_store<T, N>(g, bufU, 5 + NC, L, uz, 0, y, zt, hf);
  }
}

// ---------------------------------------------------------------------------
// K4: z forward FFT + derivative combination + cylinder pack into ub (TB_F)
// grid (n, ceil(kxn/k4_xt)).  Output slots: 0 = d/dx(u^2-v^2)+d/dz(uw) partial,
// 1 = uv, 2 = d/dx(uw)+d/dz(w^2-v^2), 3 = vw (y derivatives added in K5).
// ---------------------------------------------------------------------------
template <typename T, int N, int XT>
__device__ __forceinline__ void zfwd_load(const Geo& g, const C2<T>* __restrict__ uz, int slot, int y0, int ny,
                                          int x0, int nl, C2<T>* buf, int L) {
  // lines l = yy*nl + xl, rows y0+yy, columns x0+xl; full tiles (nl = XT)
  // take the loop with compile-time divisors
  constexpr int TZ = Tiles<T>::TZ;
  auto copy = [&](auto nlc, const C2<T>* src, C2<T>* b) {
    constexpr int NLC = decltype(nlc)::value;
    const unsigned w = (NLC > 0 ? NLC : nl) * TZ;
    const unsigned cnt = (NLC > 0 ? NLC : nl) * N;
    for (unsigned e = threadIdx.x; e < cnt; e += blockDim.x) {
      const unsigned zt = e / w, rem = e % w, l = rem / TZ, zz = rem % TZ;
      cp_async_elem(b + l * L + pad32(zt * TZ + zz), src + ((size_t)zt * g.kxn + l) * TZ + zz);
    }
  };
  for (int yy = 0; yy < ny; yy++) {
    const size_t vbase = ((size_t)slot * N + y0 + yy) * g.nzt;
    const C2<T>* src = uz + (vbase * g.kxn + x0) * TZ;
    C2<T>* b = buf + yy * nl * L;
    if (nl == XT)
      copy(std::integral_constant<int, XT>(), src, b);
    else
      copy(std::integral_constant<int, 0>(), src, b);
  }
}

template <typename T, int N, int MODE, int XT>
__device__ __forceinline__ void zfwd_store(const Geo& g, const C2<T>* s0, const C2<T>* s1, int L,
                                           C2<T>* __restrict__ ub, int slot, int y0, int /*ny*/, int x0, int x1,
                                           T b11, T b33) {
  constexpr int ny = Tiles<T>::YT4;
  // the ny rows of one block column are adjacent in ub: write them together
  using C = C2<T>;
  constexpr int TB = Tiles<T>::TBL_F;   // runs of the forward ub layout
  const int nl = x1 - x0;
  const int abeg = __ldg(g.colstart + x0), aend = __ldg(g.colstart + x1);
  const int as = abeg - (abeg % TB);                      // first block boundary
  const int cnt = ((aend - as + TB - 1) / TB) * TB * ny;  // whole blocks x rows
  C* dst = ub + (size_t)slot * ubf_var_elems<T>(g.nab_f, N);
  // column starts of the XT lines: x and z of a cylinder index follow from
  // them (column x0 + j holds kz = 0..kc then -kc..-1)
  int csr[XT + 1];
#pragma unroll
  for (int j = 0; j <= XT; j++) csr[j] = __ldg(g.colstart + min(x0 + j, g.kxn));
  for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
    // e -> (block q, row yy, column a): the ny rows of a block are adjacent
    // in memory, so consecutive threads write consecutive addresses
    const int q = e / (TB * ny), r = e % (TB * ny);
    const int yy = r / TB, a = as + q * TB + r % TB;
    if (a < abeg || a >= aend) continue;
    int lx = 0, c0 = csr[0], c1 = csr[1];
#pragma unroll
    for (int j = 1; j < XT; j++)
      if (a >= csr[j]) { lx = j; c0 = csr[j]; c1 = csr[j + 1]; }
    const int kc = (c1 - c0 - 1) / 2, ia = a - c0;
    const int x = x0 + lx, z = ia <= kc ? ia : ia + N - (2 * kc + 1), l = yy * nl + lx;
    const int i = l * L + pad32(z);
    C out;
    if constexpr (MODE == 0) {          // i kx P1 + i b33 kz P5   (s1 = P1, s0 = P5)
      const T kx = T(x), bk3 = b33 * T(kwave<N>(z));
      const C p1 = s1[i], p5 = s0[i];
      out = cmk<C>(-kx * p1.y - bk3 * p5.y, kx * p1.x + bk3 * p5.x);
    } else if constexpr (MODE == 1) {   // i b11 kx P5 + i kz P3   (s1 = P3, s0 = P5)
      const T bk1 = b11 * T(x), kz = T(kwave<N>(z));
      const C p3 = s1[i], p5 = s0[i];
      out = cmk<C>(-bk1 * p5.y - kz * p3.y, bk1 * p5.x + kz * p3.x);
    } else if constexpr (MODE == 2) {
      out = s0[i];
    } else if constexpr (MODE == 3) {
      out = s1[i];
    } else {                            // MODE 4: s0 to this slot and s1 to slot + 2
      out = s0[i];
      dst[2 * ubf_var_elems<T>(g.nab_f, N) + ((size_t)((unsigned)a / TB) * N + y0 + yy) * TB + ((unsigned)a % TB)] =
          s1[i];
    }
    dst[((size_t)((unsigned)a / TB) * N + y0 + yy) * TB + ((unsigned)a % TB)] = out;
  }
}

// K4 with register-fed transforms (the FP32 and FP64 stage kernels): pass 0
// of every z transform takes its operands straight from uz, and the last pass
// of P1, P3, P2, P4 (and of the scalar term) writes the cylinder entries of ub
// from registers (consecutive z of a warp are consecutive cylinder indices),
// so shared memory carries only the exchanges between passes and the P5
// lines that the derivative combinations of P1 and P3 read.
// Phase 1: P5, P1, P3 (P5's last pass in shared memory; then P1 -> ub slot 0,
// P3 -> slot 2); phase 2: P2 -> slot 1, P4 -> slot 3 (uz slot 5 -> ub slot 4
// with a scalar).  Field f of x line xl is line f nl + xl of its phase.
template <typename T, int N, int NC, int THREADS>
__device__ __forceinline__ void zfwd_fused(const Geo& g, const C2<T>* __restrict__ uz, C2<T>* __restrict__ ub,
                                           C2<T>* buf, const C2<T>* tw, int y, int x0, int nl, T b11, T b33) {
  using C = C2<T>;
  using PL = FFTPlan<T, N>;
  static_assert(Tiles<T>::YT4 == 1, "one y row per block");
  static_assert(PL::NPASS >= 2, "load and store passes must differ");
  constexpr int TZ = Tiles<T>::TZ, TB = Tiles<T>::TBL_F, L = LS<N>::value;
  constexpr size_t zstride = (size_t)kxn_of(N) * TZ;   // g.kxn, as a constant
  const size_t var = ubf_var_elems<T>(g.nab_f, N);
  // uz field `slot` of x line x0 + xl at row y: entry z at (z / TZ) zstride + z % TZ
  struct In { const C* src; };
  auto in_line = [&](int slot, int xl) {
    return In{uz + ((((size_t)slot * N + y) * g.nzt) * g.kxn + x0 + xl) * TZ};
  };
  auto fetch = [&](const In& s, int z) { return __ldg(s.src + ((unsigned)z / TZ) * zstride + (unsigned)z % TZ); };
  auto nofix = [](const In&, int, C v) { return v; };
  // ub slot of x line x0 + xl: column x holds kz = 0..kc then -kc..-1 from
  // cylinder index c0 (mpisetup.f:322-357); mode 0: i kx P1 + i b33 kz P5,
  // mode 1: i b11 kx P5 + i kz P3, mode 2: the value itself
  struct Out { C* dst; const C* p5; int x, c0, kc, mode; };
  auto out_line = [&](int slot, int xl, int mode) {
    const int c0 = __ldg(g.colstart + x0 + xl);
    return Out{ub + (size_t)slot * var, buf + (size_t)xl * L, x0 + xl, c0,
               (__ldg(g.colstart + x0 + xl + 1) - c0 - 1) / 2, mode};
  };
  auto store = [&](const Out& s, int base, const C* v, auto Rc, auto NSc) {
    constexpr int R = decltype(Rc)::value, NS = decltype(NSc)::value;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int z = base + r * NS;
      if (z > s.kc && z < N - s.kc) continue;
      C out = v[r];
      if (s.mode == 0) {
        const T kx = T(s.x), bk3 = b33 * T(kwave<N>(z));
        const C p5 = s.p5[pad32(z)];
        out = cmk<C>(-kx * v[r].y - bk3 * p5.y, kx * v[r].x + bk3 * p5.x);
      } else if (s.mode == 1) {
        const T bk1 = b11 * T(s.x), kz = T(kwave<N>(z));
        const C p5 = s.p5[pad32(z)];
        out = cmk<C>(-bk1 * p5.y - kz * v[r].y, bk1 * p5.x + kz * v[r].x);
      }
      const int a = s.c0 + (z <= s.kc ? z : z - N + 2 * s.kc + 1);
      s.dst[((size_t)((unsigned)a / TB) * N + y) * TB + ((unsigned)a % TB)] = out;
    }
  };
  // phase 1
  fft_pass0_load<T, N, THREADS>(
      buf, 3 * nl, L, [&](int l) { return in_line(l < nl ? 4 : (l < 2 * nl ? 0 : 2), l % nl); }, fetch, nofix);
  cp_async_wait_all();
  __syncthreads();
  fft_passes_until<T, N, THREADS, 1, PL::NPASS - 1>(buf, 3 * nl, L, tw);
  fft_passes_until<T, N, THREADS, PL::NPASS - 1, PL::NPASS>(buf, nl, L, tw);
  __syncthreads();   // P5 lines complete
  fft_pass_last_store<T, N, THREADS>(buf + (size_t)nl * L, 2 * nl, L, tw,
                                     [&](int l) { return l < nl ? out_line(0, l, 0) : out_line(2, l - nl, 1); },
                                     store);
  __syncthreads();   // every line of phase 1 read
  // phase 2
  constexpr int NV2 = 2 + NC;
  fft_pass0_load<T, N, THREADS>(
      buf, NV2 * nl, L, [&](int l) { return in_line(l < nl ? 1 : (l < 2 * nl ? 3 : 5), l % nl); }, fetch, nofix);
  __syncthreads();
  fft_passes_until<T, N, THREADS, 1, PL::NPASS - 1>(buf, NV2 * nl, L, tw);
  fft_pass_last_store<T, N, THREADS>(
      buf, NV2 * nl, L, tw,
      [&](int l) { return out_line(l < nl ? 1 : (l < 2 * nl ? 3 : 4), l % nl, 2); }, store);
}

// XTO > 0: XTO x lines per block instead of k4_xt (ensemble tuner)
template <typename T, int N, int NC = 0, bool TCM = false, int XTO = 0>
__global__ void __launch_bounds__(K4LaunchX<T, N, (XTO > 0 ? XTO : k4_xt(sizeof(T) == 8, N)), TCM>::THREADS,
                                  K4LaunchX<T, N, (XTO > 0 ? XTO : k4_xt(sizeof(T) == 8, N)), TCM>::MINB)
k_zfwd(Geo g, const C2<T>* __restrict__ uz, C2<T>* __restrict__ ub, const C2<T>* __restrict__ tw_g,
       T b11, T b33, TcArgs tca = TcArgs()) {
  // NC = 1: the scalar advection term (uz slot 5) goes to ub slot 4 without
  // derivatives (transform.f: i2f = 4+nc)
  // grid (n / YT4, ceil(kxn / XT)): YT4 adjacent y rows x XT x lines
  using C = C2<T>;
  constexpr int XT = XTO > 0 ? XTO : k4_xt(sizeof(T) == 8, N), YT = Tiles<T>::YT4, NLT = XT * YT;
  static_assert(!TCM || NLT >= 4, "an operand tile overlays four lines of s0 or s1");
  constexpr int THREADS = K4LaunchX<T, N, XT, TCM>::THREADS;
  constexpr int L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* s0 = tw + FFTPlan<T, N>::TWSIZE;
  C* s1 = s0 + NLT * L;
  load_twiddles<T, N>(tw, tw_g);
  // grid (n / YT4, ceil(kxn / XT), boxes)
  const int y0 = blockIdx.x * YT, x0 = blockIdx.y * XT, box = blockIdx.z;
  uz += box * g.zbox;
  ub += box * g.bbox;
  const int x1 = min(x0 + XT, g.kxn);
  const int nl = x1 - x0;
  if constexpr (!TCM) {
    zfwd_fused<T, N, NC, THREADS>(g, uz, ub, s0, tw, y0, x0, nl, b11, b33);
  } else {
    // tensor-core form: rounds of two fields through shared memory
    constexpr int NCOL = tc_cols(2 * NLT);
    tc::Work w;
    tc_begin<NCOL>(w, reinterpret_cast<unsigned char*>(s1 + NLT * L), tca);
    const int nt = nl * YT;
    // round 1: P5 -> s0, P1 -> s1
    zfwd_load<T, N, XT>(g, uz, 4, y0, YT, x0, nl, s0, L);
    zfwd_load<T, N, XT>(g, uz, 0, y0, YT, x0, nl, s1, L);
    cp_async_wait_all();
    __syncthreads();
    if (nl == XT) {
      lines_fft<T, N, THREADS, TCM>(s0, 2 * NLT, L, tw, w);
    } else {
      lines_fft<T, N, THREADS, TCM>(s0, nt, L, tw, w);
      lines_fft<T, N, THREADS, TCM>(s1, nt, L, tw, w);
    }
    zfwd_store<T, N, 0, XT>(g, s0, s1, L, ub, 0, y0, YT, x0, x1, b11, b33);
    __syncthreads();
    // round 2: P3 -> s1
    zfwd_load<T, N, XT>(g, uz, 2, y0, YT, x0, nl, s1, L);
    cp_async_wait_all();
    __syncthreads();
    lines_fft<T, N, THREADS, TCM>(s1, nt, L, tw, w);
    zfwd_store<T, N, 1, XT>(g, s0, s1, L, ub, 2, y0, YT, x0, x1, b11, b33);
    __syncthreads();
    // round 3: P2 -> s0, P4 -> s1
    zfwd_load<T, N, XT>(g, uz, 1, y0, YT, x0, nl, s0, L);
    zfwd_load<T, N, XT>(g, uz, 3, y0, YT, x0, nl, s1, L);
    cp_async_wait_all();
    __syncthreads();
    if (nl == XT) {
      lines_fft<T, N, THREADS, TCM>(s0, 2 * NLT, L, tw, w);
    } else {
      lines_fft<T, N, THREADS, TCM>(s0, nt, L, tw, w);
      lines_fft<T, N, THREADS, TCM>(s1, nt, L, tw, w);
    }
    // P2 -> ub slot 1 and P4 -> ub slot 3 in one pass over the cylinder indices
    zfwd_store<T, N, 4, XT>(g, s0, s1, L, ub, 1, y0, YT, x0, x1, b11, b33);
    if constexpr (NC > 0) {
      __syncthreads();
      zfwd_load<T, N, XT>(g, uz, 5, y0, YT, x0, nl, s1, L);
      cp_async_wait_all();
      __syncthreads();
      lines_fft<T, N, THREADS, TCM>(s1, nt, L, tw, w);
      zfwd_store<T, N, 3, XT>(g, s0, s1, L, ub, 4, y0, YT, x0, x1, b11, b33);
    }
    tc::teardown<NCOL>(w);
  }
}

// ---------------------------------------------------------------------------
// K5: y forward FFT + wavespace closure + proc4a (kstep 1) / proc4b (kstep 2)
// grid (nab_f): one block = one ub block of TB_F columns
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void project3(C2<T>& u1, C2<T>& u2, C2<T>& u3, T kx, T ky, T kz,
                                         T b11, T b22, T b33) {
  using C = C2<T>;
  const T bk1 = b11 * kx, bk3 = b33 * kz, bkk3 = bk3 * kz;
  const T bk12 = bk1 * kx + b22 * (ky * ky);
  const T den = bk12 + bkk3;
  const T rden = T(1) / den;
  const T c2 = b22 * ky;
  const C s = cmk<C>(bk1 * u1.x + c2 * u2.x + bk3 * u3.x, bk1 * u1.y + c2 * u2.y + bk3 * u3.y);
  const C psi = cmk<C>(-(s.x * rden), -(s.y * rden));
  u1 = cmk<C>(u1.x + kx * psi.x, u1.y + kx * psi.y);
  u2 = cmk<C>(u2.x + ky * psi.x, u2.y + ky * psi.y);
  u3 = cmk<C>(u3.x + kz * psi.x, u3.y + kz * psi.y);
}

template <typename T, int N, int KSTEP, int NC = 0, bool TCM = false>
__global__ void __launch_bounds__(K5Launch<T, N, NC>::THREADS)
k_yfwd(Geo g, StageTables<T> st_all, const C2<T>* __restrict__ ub, C2<T>* __restrict__ u,
       C2<T>* __restrict__ un, const C2<T>* __restrict__ tw_g, double* __restrict__ efkz, TcArgs tca = TcArgs(),
       C2<T>* __restrict__ racc = nullptr) {
  // KSTEP = 11 .. 14: the RK4 sub-stages advanc_1 .. advanc_4
  // (homogeneous/advanc_1.f .. advanc_4.f, -DRKFOUR), velocity only (NC = 0);
  // racc is their accumulator u1 (comp_set.f:72):
  //   11: racc = f (un + w/3), u = f (un + w), f = xfac yfac zfac; u
  //       projected; forcing (with efkz) added to u
  //   12, 13: racc += w*2/3, u = un + w (12) or un + w*2 (13); u projected;
  //       forcing added to u
  //   14: racc += w*1/3, projected; un = u = racc, mean mode zeroed (the
  //       forcing that advanc_4.f adds to u is overwritten by that copy)
  // grid (nab_f, boxes); forcing (efkz) is for single boxes only.
  // KSTEP = 0: transfer spectrum only (trfsp.f:62-83): the shell sums of
  // tfact Re(conj(un) . w) go to efkz[n/2] (shell ik = int(|k|/st.tdk + 1.5));
  // u and un are not written.
  const int box = blockIdx.y;
  const StageTables<T> st = st_all.at_box(box);
  ub += box * g.bbox;
  u += box * g.sbox;
  un += box * g.sbox;
  // NC = 1: ub slot 4 is the scalar advection term; the scalar is un-shifted
  // (wavespace_module.f:344-357) and advanced with the diffusivity factors
  // xdif ydif zdif (proc4a.f:508-522, proc4b.f:69-75), without projection
  using C = C2<T>;
  constexpr int TB = Tiles<T>::TB_F;
  constexpr int NVF = 4 + NC;
  constexpr int THREADS = K5Launch<T, N, NC>::THREADS;
  constexpr int L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* buf = tw + FFTPlan<T, N>::TWSIZE;   // [4][TB] lines
  double* thist = reinterpret_cast<double*>(buf + NVF * TB * L);   // KSTEP = 0: [n/2] shells
  load_twiddles<T, N>(tw, tw_g);
  if constexpr (KSTEP == 0)
    for (int i = threadIdx.x; i < N / 2; i += THREADS) thist[i] = 0.0;
  const int at = blockIdx.x, a0 = at * TB;
  for (int v = 0; v < NVF; v++) {
    constexpr int TBL = Tiles<T>::TBL_F, R = TBL / TB;
    const C* src = ub + (size_t)v * ubf_var_elems<T>(g.nab_f, N) + (size_t)(at / R) * N * TBL + (at % R) * TB;
    for (int e = threadIdx.x; e < TB * N; e += THREADS) {
      const int y = e / TB, l = e % TB;
      cp_async_elem(buf + (v * TB + l) * L + pad32(y), src + y * TBL + l);
    }
  }
  const size_t vs = (size_t)g.xz_tot * N;
  // the old state un of this thread's points
  constexpr int PER = (TB * N + THREADS - 1) / THREADS;
  C nb[PER][3 + NC];
  auto load_un = [&]() {
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int e = threadIdx.x + q * THREADS;
      const int l = e / N, y = e % N, a = a0 + l;
      if (e < TB * N && a < g.xz_tot && mask_ok(g, a, y, N)) {
        const size_t o = (size_t)a * N + y;
#pragma unroll
        for (int v = 0; v < 3 + NC; v++) nb[q][v] = un[v * vs + o];
      }
    }
  };
  static_assert(!TCM || KSTEP != 0, "the transfer spectrum keeps the FP32 transform");
  constexpr int NCOL = tc_cols(NVF * TB);
  tc::Work w;
  if constexpr (TCM) tc_begin<NCOL>(w, reinterpret_cast<unsigned char*>(buf + NVF * TB * L), tca);
  cp_async_wait_all();
  __syncthreads();
  lines_fft<T, N, THREADS, TCM>(buf, NVF * TB, L, tw, w);
  if constexpr (TCM) tc::teardown<NCOL>(w);
  // issued together after the transform (registers are free again), so each
  // thread waits once for all of its points
  load_un();
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int e = threadIdx.x + q * THREADS;
    if (e >= TB * N) break;
    const int l = e / N, y = e % N, a = a0 + l;
    if (a >= g.xz_tot) continue;
    const size_t o = (size_t)a * N + y;
    if (!mask_ok(g, a, y, N)) {
      if constexpr (KSTEP != 0) {
        u[o] = cmk<C>(0, 0);
        u[vs + o] = cmk<C>(0, 0);
        u[2 * vs + o] = cmk<C>(0, 0);
        if constexpr (NC > 0) u[3 * vs + o] = cmk<C>(0, 0);
      }
      continue;
    }
    const int x = __ldg(g.ax + a), z = __ldg(g.az + a);
    const int iky = kwave<N>(y), ikz = kwave<N>(z);
    const T kx = T(x), ky = T(iky), kz = T(ikz);
    const int i = pad32(y);
    const C V1 = buf[(0 * TB + l) * L + i], V2 = buf[(1 * TB + l) * L + i];
    const C V3 = buf[(2 * TB + l) * L + i], V4 = buf[(3 * TB + l) * L + i];
    // wavespace_vel.f:165-169
    const C sxz = cmul(__ldg(st.sz + z), __ldg(st.sx + x));
    const C s = cconj(cmul(sxz, __ldg(st.sy + y)));
    const C sxyz = cmk<C>(-st.norm * s.x, -st.norm * s.y);
    const T tb = st.b22 * ky;
    const C ut1 = cmk<C>(-tb * sxyz.y, tb * sxyz.x);
    C w1 = cadd(cmul(sxyz, V1), cmul(ut1, V2));
    const C si = cmk<C>(-sxyz.y, sxyz.x);
    const T bk1 = st.b11 * kx, bk3 = st.b33 * kz;
    C w2 = cmul(si, cmk<C>(bk1 * V2.x + bk3 * V4.x, bk1 * V2.y + bk3 * V4.y));
    C w3 = cadd(cmul(sxyz, V3), cmul(ut1, V4));
    const bool k0 = (a == 0 && y == 0);
    C n1 = nb[q][0], n2 = nb[q][1], n3 = nb[q][2];
    if constexpr (KSTEP == 0) {
      const double term = ((double)n1.x * w1.x + (double)n1.y * w1.y) + ((double)n2.x * w2.x + (double)n2.y * w2.y) +
                          ((double)n3.x * w3.x + (double)n3.y * w3.y);
      const double ksq = (double)st.b11 * x * x + (double)st.b22 * iky * iky + (double)st.b33 * ikz * ikz;
      const int ik = (int)(sqrt(ksq) / st.tdk + 1.5);
      if (ik >= 1 && ik <= N / 2) atomicAdd(thist + ik - 1, term * (x == 0 ? 1.0 : 2.0));
      continue;
    }
    C u1, u2, u3;
    constexpr bool RK4 = KSTEP >= 11;
    C r1 = cmk<C>(0, 0), r2 = cmk<C>(0, 0), r3 = cmk<C>(0, 0);
    if constexpr (RK4) {
      static_assert(NC == 0, "RK4 advances the velocity only");
      if constexpr (KSTEP == 11) {
        const T f = __ldg(st.xfac + x) * __ldg(st.yfac + y) * __ldg(st.zfac + z);
        r1 = cscale(f, cadd(n1, cmk<C>(w1.x / T(3), w1.y / T(3))));
        r2 = cscale(f, cadd(n2, cmk<C>(w2.x / T(3), w2.y / T(3))));
        r3 = cscale(f, cadd(n3, cmk<C>(w3.x / T(3), w3.y / T(3))));
        u1 = cscale(f, cadd(n1, w1));
        u2 = cscale(f, cadd(n2, w2));
        u3 = cscale(f, cadd(n3, w3));
      } else {
        r1 = racc[o];
        r2 = racc[vs + o];
        r3 = racc[2 * vs + o];
        constexpr T cw = KSTEP == 14 ? T(1) : T(2);
        r1 = cadd(r1, cmk<C>(w1.x * cw / T(3), w1.y * cw / T(3)));
        r2 = cadd(r2, cmk<C>(w2.x * cw / T(3), w2.y * cw / T(3)));
        r3 = cadd(r3, cmk<C>(w3.x * cw / T(3), w3.y * cw / T(3)));
        if constexpr (KSTEP == 14) {
          u1 = r1; u2 = r2; u3 = r3;
        } else {
          constexpr T cu = KSTEP == 12 ? T(1) : T(2);
          u1 = cadd(n1, cmk<C>(w1.x * cu, w1.y * cu));
          u2 = cadd(n2, cmk<C>(w2.x * cu, w2.y * cu));
          u3 = cadd(n3, cmk<C>(w3.x * cu, w3.y * cu));
        }
      }
    } else if constexpr (KSTEP == 1) {
      // proc4a.f:427, 479-486
      const T f = k0 ? T(1) : __ldg(st.xfac + x) * __ldg(st.yfac + y) * __ldg(st.zfac + z);
      u1 = cscale(f, cmk<C>(n1.x + T(2) * w1.x, n1.y + T(2) * w1.y));
      u2 = cscale(f, cmk<C>(n2.x + T(2) * w2.x, n2.y + T(2) * w2.y));
      u3 = cscale(f, cmk<C>(n3.x + T(2) * w3.x, n3.y + T(2) * w3.y));
      n1 = cscale(f, cadd(n1, w1));
      n2 = cscale(f, cadd(n2, w2));
      n3 = cscale(f, cadd(n3, w3));
    } else {
      // proc4b.f:54-58
      u1 = cadd(n1, w1);
      u2 = cadd(n2, w2);
      u3 = cadd(n3, w3);
    }
    if (!k0) project3<T>(u1, u2, u3, kx, ky, kz, st.b11, st.b22, st.b33);
    // Eswaran-Pope forcing (proc4a.f:588-651, proc4b.f:118-163; advanc_1.f:164-216)
    constexpr bool FIRST = KSTEP == 1 || KSTEP == 11;
    if (KSTEP != 14 && st.forc != nullptr && x < st.kfor) {
      const int kf = st.kfor, k2 = st.k2fo;
      int izi = (ikz >= 0 && ikz < kf) ? ikz : ((ikz < 0 && ikz > -kf) ? ikz + k2 : -1);
      int iyi = (iky >= 0 && iky < kf) ? iky : ((iky < 0 && iky > -kf) ? iky + k2 : -1);
      if (izi >= 0 && iyi >= 0) {
        bool add = true;
        double rks = 0.0;
        if constexpr (FIRST) {
          rks = (double)x * x * (double)st.b11 + (double)iky * iky * (double)st.b22 +
                (double)ikz * ikz * (double)st.b33;
          add = rks <= st.kforce2;
        }
        if (add) {
          const size_t fo = ((size_t)izi * k2 + iyi) * kf + x;
          const size_t fs = (size_t)kf * k2 * k2;
          const C f1 = st.forc[fo], f2 = st.forc[fs + fo], f3 = st.forc[2 * fs + fo];
          if constexpr (FIRST) {
            if (efkz != nullptr) {
              const int kk = (int)(sqrt(rks) + 1.5);
              const double tf = (x == 0) ? 1.0 : 2.0;
              const double e1 = (double)u1.x * f1.x + (double)u1.y * f1.y;
              const double e2 = (double)u2.x * f2.x + (double)u2.y * f2.y;
              const double e3 = (double)u3.x * f3.x + (double)u3.y * f3.y;
              atomicAdd(efkz + (kk - 1) * 3 + 0, 2. * e1 * tf * (double)st.b11);
              atomicAdd(efkz + (kk - 1) * 3 + 1, 2. * e2 * tf * (double)st.b22);
              atomicAdd(efkz + (kk - 1) * 3 + 2, 2. * e3 * tf * (double)st.b33);
            }
          }
          u1 = cadd(u1, f1);
          u2 = cadd(u2, f2);
          u3 = cadd(u3, f3);
        }
      }
    }
    if constexpr (NC > 0) {
      const C V5 = buf[(4 * TB + l) * L + i];
      const C w4 = cmul(sxyz, V5);
      C n4 = nb[q][3], u4;
      if constexpr (KSTEP == 1) {
        const T fs = __ldg(st.xdif + x) * __ldg(st.ydif + y) * __ldg(st.zdif + z);
        u4 = cscale(fs, cmk<C>(n4.x + T(2) * w4.x, n4.y + T(2) * w4.y));
        n4 = cscale(fs, cadd(n4, w4));
      } else {
        u4 = cadd(n4, w4);
        if (k0) u4 = cmk<C>(0, 0);
        n4 = u4;
      }
      u[3 * vs + o] = u4;
      un[3 * vs + o] = n4;
    }
    if constexpr (KSTEP == 2 || KSTEP == 14) {
      if (k0) {
        u1 = u2 = u3 = cmk<C>(0, 0);
      }
      n1 = u1; n2 = u2; n3 = u3;
    }
    u[o] = u1; u[vs + o] = u2; u[2 * vs + o] = u3;
    if constexpr (RK4 && KSTEP != 14) {
      racc[o] = r1; racc[vs + o] = r2; racc[2 * vs + o] = r3;
    } else {
      un[o] = n1; un[vs + o] = n2; un[2 * vs + o] = n3;
    }
  }
  if constexpr (KSTEP == 0) {
    __syncthreads();
    for (int i = threadIdx.x; i < N / 2; i += THREADS)
      if (thist[i] != 0.0) atomicAdd(efkz + i, thist[i]);
  }
}

// ---------------------------------------------------------------------------
// Spline coefficients: backward x transform of the prefiltered field (pairs
// of z lines as in K3) and store of (c_u, c_v, c_w, 0) per grid point into
// bs[y][z][x] (vector of 4).  grid (nzt, n).
// ---------------------------------------------------------------------------
template <typename T> struct V4T;
template <> struct V4T<float> { using type = float4; };
template <> struct V4T<double> { using type = double4; };

template <typename T, int N>
__global__ void __launch_bounds__(Launch<T, N, 2 * Tiles<T>::TZ>::THREADS)
k_xspline(Geo g, const C2<T>* __restrict__ uz, typename V4T<T>::type* __restrict__ bs,
          const C2<T>* __restrict__ tw_g) {
  using C = C2<T>;
  using V4 = typename V4T<T>::type;
  constexpr int TZ = Tiles<T>::TZ, NPAIR = TZ / 2;
  constexpr int THREADS = Launch<T, N, 2 * TZ>::THREADS;
  constexpr int L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* bufU = tw + FFTPlan<T, N>::TWSIZE;
  load_twiddles<T, N>(tw, tw_g);
  const int zt = blockIdx.x, y = blockIdx.y;
  const int kxn = g.kxn;
  if constexpr (XFuse<T, N>::value) {
    xchain_load_pass0<T, N, 3, THREADS>(g, uz, 0, y, zt, bufU, L);
    cp_async_wait_all();
    __syncthreads();
    fft_passes<T, N, THREADS, 1>(bufU, 3 * NPAIR, L, tw);
    __syncthreads();
  } else {
    for (int e = threadIdx.x; e < 3 * NPAIR * N; e += THREADS) {
      const int k = e % N;
      if (k >= kxn && k <= N - kxn) bufU[(e / N) * L + pad32(k)] = cmk<C>(0, 0);
    }
    xchain_pack<T, N, 3, THREADS>(g, uz, 0, y, zt, bufU, L);
    cp_async_wait_all();
    __syncthreads();
    fft_lines<T, N, THREADS>(bufU, 3 * NPAIR, L, tw);
  }
  // buffer = conj(a + i b): line z = 2p is re, line 2p+1 is -im
  for (int e = threadIdx.x; e < TZ * N; e += THREADS) {
    const int zz = e / N, x = e % N, p = zz / 2;
    const int i = p * L + pad32(x);
    const C U = bufU[i], V = bufU[NPAIR * L + i], W = bufU[2 * NPAIR * L + i];
    V4 c;
    if (zz & 1) { c.x = -U.y; c.y = -V.y; c.z = -W.y; } else { c.x = U.x; c.y = V.x; c.z = W.x; }
    c.w = 0;
    bs[((size_t)y * N + zt * TZ + zz) * N + x] = c;
  }
}

// ---------------------------------------------------------------------------
// Velocity-gradient moments (vgmomt.f:50-143): x inverse of the two gradient
// fields of uz slots 0 and 1, then the sums of g^m, m = 1..8, in FP64; each
// block writes its 16 partial sums, k_moments_reduce adds them in a fixed
// order.  grid (nzt, n).
// ---------------------------------------------------------------------------
template <typename T, int N>
struct KMomLaunch : Launch<T, N, 2 * (Tiles<T>::TZ / 2)> {
  static constexpr size_t SMEM =
      sizeof(C2<T>) * (FFTPlan<T, N>::TWSIZE + (size_t)2 * (Tiles<T>::TZ / 2) * LS<N>::value);
};

template <typename T, int N>
__global__ void __launch_bounds__(KMomLaunch<T, N>::THREADS)
k_xmoments(Geo g, const C2<T>* __restrict__ uz, const C2<T>* __restrict__ tw_g, double* __restrict__ partial) {
  using C = C2<T>;
  constexpr int TZ = Tiles<T>::TZ, NPAIR = TZ / 2;
  constexpr int THREADS = KMomLaunch<T, N>::THREADS;
  static_assert(THREADS % 32 == 0, "the reduction uses whole warps");
  constexpr int L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* bufU = tw + FFTPlan<T, N>::TWSIZE;
  __shared__ double red[THREADS / 32 + 1][16];
  load_twiddles<T, N>(tw, tw_g);
  const int zt = blockIdx.x, y = blockIdx.y, kxn = g.kxn;
  for (int e = threadIdx.x; e < 2 * NPAIR * N; e += THREADS) {
    const int k = e % N;
    if (k >= kxn && k <= N - kxn) bufU[(e / N) * L + pad32(k)] = cmk<C>(0, 0);
  }
  xchain_pack<T, N, 2, THREADS>(g, uz, 0, y, zt, bufU, L);
  cp_async_wait_all();
  __syncthreads();
  fft_lines<T, N, THREADS>(bufU, 2 * NPAIR, L, tw);
  // buffer = conj(a + i b): real line z = 2p is re, 2p+1 is -im
  double s[16];
#pragma unroll
  for (int m = 0; m < 16; m++) s[m] = 0.0;
  for (int e = threadIdx.x; e < TZ * N; e += THREADS) {
    const int zz = e / N, x = e % N, p = zz / 2;
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const C z = bufU[(f * NPAIR + p) * L + pad32(x)];
      const double v = (zz & 1) ? -(double)z.y : (double)z.x, sq = v * v;
      s[8 * f + 0] += v;
      s[8 * f + 1] += sq;
      s[8 * f + 2] += sq * v;
      s[8 * f + 3] += sq * sq;
      s[8 * f + 4] += sq * sq * v;
      s[8 * f + 5] += sq * sq * sq;
      s[8 * f + 6] += sq * sq * sq * v;
      s[8 * f + 7] += sq * sq * sq * sq;
    }
  }
  // fixed-order block reduction: warps by shuffles, then warp sums in order
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < 16; m++) {
    double v = s[m];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][m] = v;
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    double v = 0.0;
    for (int w = 0; w < THREADS / 32; w++) v += red[w][threadIdx.x];
    partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 16 + threadIdx.x] = v;
  }
}

// out[m] = (sum over blocks of partial[.][m]) * scale, one block per m
static __global__ void __launch_bounds__(256) k_moments_reduce(const double* __restrict__ partial, long long nblocks,
                                                        double scale, double* __restrict__ out) {
  __shared__ double red[256];
  const int m = blockIdx.x;
  double v = 0.0;
  for (long long b = threadIdx.x; b < nblocks; b += 256) v += partial[b * 16 + m];
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[m] = red[0] * scale;
}

// ---------------------------------------------------------------------------
// Lagrangian particles: one Heun (RK2) step with two cubic-spline
// interpolations (partsp.f:231-299,405-412, rk_advpos.f:29-37,65-72,
// spcal_local.f:118-367).  Positions are FP64 in grid units (grid plane i at
// 1 + (i-1) + gsh(.,1), partsp.f:44-51).  Sixteen lanes share a particle:
// lane r gathers the 4 x-points of row (y, z) = (r/4, r%4) of the 4x4x4
// stencil, and the partial sums are reduced with warp shuffles.
// first != 0: interpolate only (first step, partsp.f:206).
// ---------------------------------------------------------------------------
// spcal_local.f:175-181, :211-231: cell index and cubic B-spline weights
// along one axis.  jloc = ipx mod n in [0, n) (the reference adds 1000 n to
// a negative ipx before its modulo), taken as fl - n floor(fl / n): exact in
// FP64 while |ipx| < 2^52 / n, so bfp has the reference's value bit for bit.
// For n = 2^k, fl / n is the exact product fl * 2^-k (2^-k built from its
// exponent bits), so the FP64 division is taken only for other n.
__device__ __forceinline__ void spline_weights(double pos, double gfn, int n, int& ib, double w[4]) {
  const double px1 = pos - gfn;
  const double px = px1 - (double)n;
  const double fl = floor(px);
  const double dn = (double)n;
  const double q = (n & (n - 1)) == 0 ? fl * __longlong_as_double((long long)(1023 - (31 - __clz(n))) << 52)
                                      : fl / dn;
  const double jloc = fl - dn * floor(q);
  const double bfp = (jloc + px) - fl;
  ib = (int)bfp;
  const double t = bfp - ib;
  const double d6 = 1. / 6., tt = 2. / 3.;
  const double ym = 1. - t, yms = ym * ym;
  w[0] = ym * yms * d6;
  w[1] = tt + 0.5 * t * (yms - 1.);
  w[3] = t * t * t * d6;
  w[2] = 1. - w[0] - w[1] - w[3];
}

// periodic index of stencil point ib + k - 1, k = 0..3 (ib in [0, n])
__device__ __forceinline__ int wrap_n(int v, int n) {
  v += (v < 0) ? n : 0;
  return v - ((v >= n) ? n : 0);
}

// spcal_local.f:234-367: the 4x4x4 stencil sum of one particle by 16 lanes,
// lane (jz, kx) summing the 4 points (jy = 0..3, jz, kx) of the stencil.  A
// warp load instruction (one jy) then reads 8 x rows of 4 points, each 64
// contiguous bytes taken by 4 adjacent lanes, for the stencils of two
// particles (lane (jy, jz) reading a row of 4 points itself made every load
// instruction touch 32 rows, holding the L1 at 85% of its throughput).
template <typename V4>
__device__ __forceinline__ void spline_interp(const V4* __restrict__ bs, int n, const double p[3],
                                              const double gfn[3], int lane16, unsigned mask16, double out[3]) {
  int ib[3];
  double wx[4], wy[4], wz[4];
  spline_weights(p[0], gfn[0], n, ib[0], wx);
  spline_weights(p[1], gfn[1], n, ib[1], wy);
  spline_weights(p[2], gfn[2], n, ib[2], wz);
  const int kx = lane16 & 3, jz = lane16 >> 2;
  // bs index ib+k (k = 1..4) holds grid point ib+k-2 (splx.f:29-35)
  const int xx = wrap_n(ib[0] + kx - 1, n), zz = wrap_n(ib[2] + jz - 1, n);
  V4 c[4];
#pragma unroll
  for (int jy = 0; jy < 4; jy++) c[jy] = bs[((size_t)wrap_n(ib[1] + jy - 1, n) * n + zz) * n + xx];
  double sx = 0, sy = 0, sz = 0;
#pragma unroll
  for (int jy = 0; jy < 4; jy++) {
    sx += wy[jy] * (double)c[jy].x;
    sy += wy[jy] * (double)c[jy].y;
    sz += wy[jy] * (double)c[jy].z;
  }
  // register selects (an indexed array would live in local memory)
  const double wxk = kx == 0 ? wx[0] : kx == 1 ? wx[1] : kx == 2 ? wx[2] : wx[3];
  const double wzj = jz == 0 ? wz[0] : jz == 1 ? wz[1] : jz == 2 ? wz[2] : wz[3];
  const double wxz = wxk * wzj;
  sx *= wxz; sy *= wxz; sz *= wxz;
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(mask16, sx, o, 16);
    sy += __shfl_xor_sync(mask16, sy, o, 16);
    sz += __shfl_xor_sync(mask16, sz, o, 16);
  }
  out[0] = sx; out[1] = sy; out[2] = sz;
}

// Heun step of rk_advpos.f (rk_advpos(1,.5,.5) then rk_advpos(2,0,.5)),
// 16 lanes per particle
template <typename T>
__global__ void __launch_bounds__(256) k_particles(const typename V4T<T>::type* __restrict__ bs, int n, long long np,
                                                   double* __restrict__ pos, double* __restrict__ vel, double g1,
                                                   double g2, double g3, double fact1, double fact2, int first) {
  const int lane16 = threadIdx.x & 15;
  const unsigned mask16 = 0xffffu << (threadIdx.x & 16);
  const long long groups = (long long)gridDim.x * (blockDim.x / 16);
  const double gfn[3] = {g1 + 1., g2 + 1., g3 + 1.};
  for (long long m = (long long)blockIdx.x * (blockDim.x / 16) + (threadIdx.x >> 4); m < np; m += groups) {
    double x[3] = {pos[m], pos[np + m], pos[2 * np + m]};
    double v[3];
    if (first) {
      spline_interp(bs, n, x, gfn, lane16, mask16, v);
    } else {
      // rk_advpos(1,.5,.5): pp7 = x + fact1 v, x = pp7 + fact2 v
      const double u0[3] = {vel[m], vel[np + m], vel[2 * np + m]};
      double h[3], xs[3], vs[3];
      for (int k = 0; k < 3; k++) { h[k] = x[k] + fact1 * u0[k]; xs[k] = h[k] + fact2 * u0[k]; }
      spline_interp(bs, n, xs, gfn, lane16, mask16, vs);
      // rk_advpos(2,0,.5): x = pp7 + fact2 v*
      for (int k = 0; k < 3; k++) x[k] = h[k] + fact2 * vs[k];
      spline_interp(bs, n, x, gfn, lane16, mask16, v);
    }
    if (lane16 == 0) {
      pos[m] = x[0]; pos[np + m] = x[1]; pos[2 * np + m] = x[2];
      vel[m] = v[0]; vel[np + m] = v[1]; vel[2 * np + m] = v[2];
    }
  }
}

// ---------------------------------------------------------------------------
// State conversion (complex double host layout <-> device precision)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_from_f64(const double2* __restrict__ src, C2<T>* __restrict__ dst, C2<T>* __restrict__ dst2,
                           size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 s = src[i];
    const C2<T> d = cmk<C2<T>>((T)s.x, (T)s.y);
    dst[i] = d;
    if (dst2) dst2[i] = d;
  }
}

template <typename T>
__global__ void k_to_f64(const C2<T>* __restrict__ src, double2* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const C2<T> s = src[i];
    dst[i] = make_double2((double)s.x, (double)s.y);
  }
}

// Full half-complex layout u(nxh, ny, nz) (column-major, nxh = n/2 + 1, the
// FFTW real-to-complex shape of a real (nx, ny, nz) array) <-> cylinder
// columns: column a = (x, z) holds every y of (x, ., z).
// Host <-> device copies of the entries inside the truncation sphere only
// (mask of masks.f: y != n/2 and min(y, n-y) <= kymax(a)), reading or writing
// pinned host memory directly (a warp per column; each column's entries are
// the runs y = 0..kym and n-kym..n-1, so a warp moves 512 contiguous bytes per
// instruction).  Columns a0..a1-1 of every variable; entries outside the
// sphere are neither read nor written.
__device__ __forceinline__ int sphere_y(int i, int kym, int n) { return i <= kym ? i : n - 2 * kym - 1 + i; }

template <typename T>
__global__ void __launch_bounds__(256) k_sphere_in(Geo g, int nv, const double2* __restrict__ h,
                                                   C2<T>* __restrict__ un, C2<T>* __restrict__ u, int a0, int a1) {
  const int n = g.n;
  const size_t vs = (size_t)g.xz_tot * n;
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int a = a0 + w0; a < a1; a += nw) {
    const int kym = __ldg(g.kymax + a), cnt = 2 * kym + 1;
    for (int v = 0; v < nv; v++) {
      const size_t base = v * vs + (size_t)a * n;
      // four independent reads in flight per thread (bus latency)
      for (int i0 = 0; i0 < cnt; i0 += 128) {
        double2 x[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int i = i0 + j * 32 + lane;
          if (i < cnt) x[j] = h[base + sphere_y(i, kym, n)];
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int i = i0 + j * 32 + lane;
          if (i < cnt) {
            const size_t e = base + sphere_y(i, kym, n);
            const C2<T> c = cmk<C2<T>>((T)x[j].x, (T)x[j].y);
            un[e] = c;
            u[e] = c;
          }
        }
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_sphere_out(Geo g, int nv, const C2<T>* __restrict__ src,
                                                    double2* __restrict__ h, int a0, int a1) {
  const int n = g.n;
  const size_t vs = (size_t)g.xz_tot * n;
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int a = a0 + w0; a < a1; a += nw) {
    const int kym = __ldg(g.kymax + a), cnt = 2 * kym + 1;
    for (int v = 0; v < nv; v++) {
      const size_t base = v * vs + (size_t)a * n;
      for (int i0 = 0; i0 < cnt; i0 += 128) {
        C2<T> c[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int i = i0 + j * 32 + lane;
          if (i < cnt) c[j] = src[base + sphere_y(i, kym, n)];
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int i = i0 + j * 32 + lane;
          if (i < cnt) h[base + sphere_y(i, kym, n)] = make_double2((double)c[j].x, (double)c[j].y);
        }
      }
    }
  }
}

template <typename T>
__global__ void k_full_to_cyl(Geo g, const double2* __restrict__ full, C2<T>* __restrict__ dst,
                              C2<T>* __restrict__ dst2) {
  const int n = g.n, nxh = n / 2 + 1;
  const size_t tot = (size_t)g.xz_tot * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(i / n), y = (int)(i % n);
    const double2 s = full[((size_t)__ldg(g.az + a) * n + y) * nxh + __ldg(g.ax + a)];
    const C2<T> d = cmk<C2<T>>((T)s.x, (T)s.y);
    dst[i] = d;
    if (dst2) dst2[i] = d;
  }
}

template <typename T>
__global__ void k_cyl_to_full(Geo g, const C2<T>* __restrict__ src, double2* __restrict__ full) {
  const int n = g.n, nxh = n / 2 + 1;
  const size_t tot = (size_t)g.xz_tot * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(i / n), y = (int)(i % n);
    const C2<T> s = src[i];
    full[((size_t)__ldg(g.az + a) * n + y) * nxh + __ldg(g.ax + a)] = make_double2((double)s.x, (double)s.y);
  }
}

}  // namespace psdns
