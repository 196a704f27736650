// psdns_host.h -- host-side helpers of libpsdns_gpu (geometry, RNG, errors).
#pragma once
#include <stdint.h>

#include <vector>

namespace psdns {

// Truncation-cylinder geometry of an n^3 box (PSDNS/mpisetup.f:307-357) and
// the spherical mask (PSDNS/masks.f:46-83) as the largest |ky| kept per column.
struct Geometry {
  int n = 0, kxn = 0, xz_tot = 0;
  std::vector<double> kx, ky, kz;   // PSDNS/init.f:15-27
  std::vector<int> cut;             // cut_z(x)
  std::vector<int> colstart;        // [kxn+1] first column a of each x
  std::vector<int> ax, az;          // per column: x index, z index (0..n-1)
  std::vector<int> kymax;           // per column: largest |ky| inside the sphere (-1: none)
};

void build_geometry(int n, Geometry& g);

// PSDNS/ranu.f + PSDNS/ranseq.f: twenty 32-bit multiplicative LCG sequences
struct Rng {
  int32_t iseq[20];
  int klast;
  int32_t iseed;
  int ifst;
  int32_t seed_input;
  void init(int32_t seed);
  void ranseq(int k);
  double ranu();
};

// PSDNS/rann2.f: Gaussian numbers by inversion of a 201-point table
struct Rann2 {
  std::vector<double> tab, dtab;   // 1-based
  double p1 = 0;
  int ntabm = 0;
  bool ready = false;
  void init();
  void draw(Rng& r, double* x, int n);
};

// Eswaran-Pope forcing (PSDNS/force.f, vfuo.f, vfiuo.f, raniuo.f)
struct EPForcing {
  int kfor = 0, k2fo = 0, nrproc = 0, n = 0, kranf1 = 5, kranf2 = 5;
  double kforce = 0, tforce = 0, epsfor = 0, tfiuo = 0, b11 = 1, b22 = 1, b33 = 1;
  double t1 = 0, t2 = 0, siga = 0;
  bool first = true;
  std::vector<double> suo, svo, velinc, w1, w2;
  std::vector<double> table;   // for(kfor,k2fo,k2fo,3), interleaved complex
  Rann2 g;
  void setup(int kfor, int nx, double kforce, double tforce, double epsfor, double tfiuo, int kranf1, int kranf2,
             double b11, double b22, double b33);
  void raniuo(Rng& r, double dt);
  void step(Rng& r, double dt, int istart);
};

int set_error(const char* fmt, ...);

// spectral-correction network (learned.cu): forward pass of nb feature rows
namespace mlp {
int forward_host(void* corr, long long nb, const float* x, float* g);
}

}  // namespace psdns
