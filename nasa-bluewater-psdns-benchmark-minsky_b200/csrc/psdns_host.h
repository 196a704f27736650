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

int set_error(const char* fmt, ...);

}  // namespace psdns
