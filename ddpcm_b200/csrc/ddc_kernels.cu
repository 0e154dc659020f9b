// ddc_kernels.cu -- sm_100a kernels of the ddCOSMO path.
//
// Conventions.  Set-defining geometry (the neighbour test, t < 1, f_i, U_i,
// the switch band) is evaluated with round-to-nearest intrinsics in the
// reference's operation order (ddcosmo.f90:310-411, 1707-1716), so the GPU
// takes the same discrete decisions as an IEEE evaluation of the reference
// loops.  Inside the hot loops the arithmetic is free to contract and to
// reorder (values only), and every reduction has a fixed order, so results
// are deterministic from run to run.
#include <climits>

#include <cub/cub.cuh>
#include <type_traits>

#include "ddc_internal.h"

namespace ddc {

#define DADD __dadd_rn
#define DSUB __dsub_rn
#define DMUL __dmul_rn
#define DDIV __ddiv_rn

__host__ __device__ constexpr int lmi(int l, int m) { return l * (l + 1) / 2 + m; }

// recurrence constants in the arithmetic type of the kernel
template <class Rl> __device__ __forceinline__ Rl cA(const YlmTables& tb, int e);
template <> __device__ __forceinline__ double cA<double>(const YlmTables& tb, int e) { return tb.A[e]; }
template <> __device__ __forceinline__ float cA<float>(const YlmTables& tb, int e) { return tb.Af[e]; }
template <class Rl> __device__ __forceinline__ Rl cB(const YlmTables& tb, int e);
template <> __device__ __forceinline__ double cB<double>(const YlmTables& tb, int e) { return tb.B[e]; }
template <> __device__ __forceinline__ float cB<float>(const YlmTables& tb, int e) { return tb.Bf[e]; }
template <class Rl> __device__ __forceinline__ Rl cK(const YlmTables& tb, int e);
template <> __device__ __forceinline__ double cK<double>(const YlmTables& tb, int e) { return tb.K[e]; }
template <> __device__ __forceinline__ float cK<float>(const YlmTables& tb, int e) { return tb.Kf[e]; }


// ---------------------------------------------------------------------------
// exact geometry helpers
// ---------------------------------------------------------------------------
// v = (c_a + r_a * s) - c_b, |v|, t = |v| / r_b   (ddcosmo.f90:378-380)
struct Rel {
  double vx, vy, vz, vv, t;
};
__device__ __forceinline__ Rel rel_exact(double4 ca, double4 g, double4 cb) {
  Rel r;
  r.vx = DSUB(DADD(ca.x, DMUL(ca.w, g.x)), cb.x);
  r.vy = DSUB(DADD(ca.y, DMUL(ca.w, g.y)), cb.y);
  r.vz = DSUB(DADD(ca.z, DMUL(ca.w, g.z)), cb.z);
  r.vv = __dsqrt_rn(DADD(DADD(DMUL(r.vx, r.vx), DMUL(r.vy, r.vy)), DMUL(r.vz, r.vz)));
  r.t = DDIV(r.vv, cb.w);
  return r;
}
// |ca + ra g - cb|^2 with the rounding steps of rel_exact; above
// rb^2 (1 + 1e-10) the point is outside sphere b by far more than the
// rounding of rel_exact's t, so t >= 1 there: chi(t) = 0 and the pair
// contributes nothing (a cheap test ahead of the square root and division)
__device__ __forceinline__ bool rel_outside(double4 ca, double4 g, double4 cb) {
  const double vx = DSUB(DADD(ca.x, DMUL(ca.w, g.x)), cb.x);
  const double vy = DSUB(DADD(ca.y, DMUL(ca.w, g.y)), cb.y);
  const double vz = DSUB(DADD(ca.z, DMUL(ca.w, g.z)), cb.z);
  const double s2 = DADD(DADD(DMUL(vx, vx), DMUL(vy, vy)), DMUL(vz, vz));
  return s2 > cb.w * cb.w * (1.0 + 1e-10);
}

// switch function chi(t) and chi'(t) for se = -1 (ddcosmo.f90:566-655)
__device__ __forceinline__ double eta5(double eta) {
  double e2 = DMUL(eta, eta);
  return DMUL(DMUL(e2, e2), eta);
}
__device__ __forceinline__ double fsw_exact(double x, double eta) {
  if (x >= 1.0) return 0.0;
  if (x <= DSUB(1.0, eta)) return 1.0;
  double a = DSUB(DMUL(15.0, eta), 12.0);
  double b = DADD(DSUB(DMUL(DMUL(10.0, eta), eta), DMUL(15.0, eta)), 6.0);
  double xm = DSUB(x, 1.0);
  double p = DMUL(DMUL(xm, xm), DSUB(1.0, x));
  double q = DADD(DADD(DMUL(DMUL(6.0, x), x), DMUL(a, x)), b);
  return DDIV(DMUL(p, q), eta5(eta));
}
__device__ __forceinline__ double dfsw_exact(double x, double eta) {
  if (x >= 1.0) return 0.0;
  if (x <= DSUB(1.0, eta)) return 0.0;
  double xm = DSUB(x, 1.0);
  double xe = DADD(xm, eta);
  return DDIV(DMUL(DMUL(DMUL(DMUL(30.0, DSUB(1.0, x)), xm), xe), xe), eta5(eta));
}
// value-only versions (contracted); same branches
__device__ __forceinline__ double fsw_fast(double x, double eta, double flow, double a, double b,
                                           double ie5) {
  if (x >= 1.0) return 0.0;
  if (x <= flow) return 1.0;
  double xm = x - 1.0;
  return (xm * xm * (1.0 - x)) * ((6.0 * x + a) * x + b) * ie5;
}

// ---------------------------------------------------------------------------
// reference spherical harmonics (init only): ylmbas ddcosmo.f90:830-895
// ---------------------------------------------------------------------------
__device__ void ylmbas_ref(const YlmTables& tb, double sx, double sy, double sz, double* basloc) {
  const int lmax = tb.lmax;
  double vplm[(DDC_MAX_LMAX + 1) * (DDC_MAX_LMAX + 1)];
  double vc[DDC_MAX_LMAX + 2], vs[DDC_MAX_LMAX + 2];
  double cthe = sz;
  double sthe = __dsqrt_rn(DSUB(1.0, DMUL(cthe, cthe)));
  if (sthe != 0.0) {
    double cphi = DDIV(sx, sthe), sphi = DDIV(sy, sthe);
    vc[0] = 1.0; vs[0] = 0.0; vc[1] = cphi; vs[1] = sphi;
    for (int m = 2; m <= lmax; m++) {
      vc[m] = DSUB(DMUL(DMUL(2.0, cphi), vc[m - 1]), vc[m - 2]);
      vs[m] = DSUB(DMUL(DMUL(2.0, cphi), vs[m - 1]), vs[m - 2]);
    }
  } else {
    for (int m = 0; m <= lmax; m++) { vc[m] = 1.0; vs[m] = 0.0; }
  }
  // polleg (ddcosmo.f90:1056-1094)
  double fact = 1.0, pmm = 1.0;
  for (int m = 0; m <= lmax; m++) {
    int ind = (m + 1) * (m + 1) - 1;
    vplm[ind] = pmm;
    if (m == lmax) break;
    double fm = (double)m;
    double pmm1 = DMUL(DMUL(cthe, DADD(DMUL(2.0, fm), 1.0)), pmm);
    vplm[ind + 2 * m + 2] = pmm1;
    double pmmo = pmm;
    for (int l = m + 2; l <= lmax; l++) {
      double fl = (double)l;
      double pll = DDIV(DSUB(DMUL(DMUL(cthe, DSUB(DMUL(2.0, fl), 1.0)), pmm1),
                             DMUL(DSUB(DADD(fl, fm), 1.0), pmm)),
                        DSUB(fl, fm));
      vplm[l * l + l + m] = pll;
      pmm = pmm1;
      pmm1 = pll;
    }
    pmm = DMUL(DMUL(-pmmo, fact), sthe);
    fact = DADD(fact, 2.0);
  }
  for (int l = 0; l <= lmax; l++) {
    int ind = l * l + l;
    basloc[ind] = DMUL(tb.facs[lmi(l, 0)], vplm[ind]);
    for (int m = 1; m <= l; m++) {
      double plm = vplm[ind + m];
      basloc[ind + m] = DMUL(DMUL(tb.facs[lmi(l, m)], plm), vc[m]);
      basloc[ind - m] = DMUL(DMUL(tb.facs[lmi(l, m)], plm), vs[m]);
    }
  }
}

__global__ void k_basis(const YlmTables tb, const double4* __restrict__ grid, double* basis,
                        double* bw) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= tb.ngrid) return;
  double4 g = grid[n];
  double* b = basis + (size_t)n * tb.nylm;
  ylmbas_ref(tb, g.x, g.y, g.z, b);
  for (int k = 0; k < tb.nylm; k++) bw[(size_t)n * tb.nylm + k] = b[k] * g.w;
}

cudaError_t launch_basis(Launch L, const YlmTables& tb, const double4* grid, double* basis,
                         double* bw) {
  k_basis<<<(tb.ngrid + 63) / 64, 64, 0, L.st>>>(tb, grid, basis, bw);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// CSR neighbour list: warp per sphere, ballot over candidates in index order
// (ddcosmo.f90:308-324); d^2 <= (r_i + r_j)^2
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool is_nb(double4 a, double4 b) {
  double dx = DSUB(a.x, b.x), dy = DSUB(a.y, b.y), dz = DSUB(a.z, b.z);
  double d2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
  double rs = DADD(a.w, b.w);
  return d2 <= DMUL(rs, rs);
}

template <bool FILL>
__global__ void k_csr(int nsph, const double4* __restrict__ sph, int* cnt, const int* inl,
                      int* nl, const int2* __restrict__ mrange) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nsph) return;
  const int i = warp;
  const double4 ci = sph[i];
  int base = FILL ? inl[i] : 0;
  // candidates: the sphere's own molecule (all spheres for a single molecule)
  const int jlo = mrange ? mrange[i].x : 0, jhi = mrange ? mrange[i].y : nsph;
  for (int j0 = jlo; j0 < jhi; j0 += 32) {
    int j = j0 + lane;
    bool nb = false;
    if (j < jhi && j != i) nb = is_nb(ci, sph[j]);
    unsigned mask = __ballot_sync(0xffffffffu, nb);
    if (FILL && nb) nl[base + __popc(mask & ((1u << lane) - 1u))] = j;
    base += __popc(mask);
  }
  if (!FILL && lane == 0) cnt[i] = base;
}

cudaError_t launch_csr_count(Launch L, int nsph, const double4* sph, int* cnt,
                             const int2* mrange) {
  k_csr<false><<<(nsph + 7) / 8, 256, 0, L.st>>>(nsph, sph, cnt, nullptr, nullptr, mrange);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_csr_fill(Launch L, int nsph, const double4* sph, const int* inl, int* nl,
                            const int2* mrange) {
  k_csr<true><<<(nsph + 7) / 8, 256, 0, L.st>>>(nsph, sph, nullptr, inl, nl, mrange);
  ++*L.launches;
  return cudaGetLastError();
}

// The same lists for one molecule from its cell groups (ddc_zfar.cu): a warp
// per sphere tests the groups' bounding spheres (a neighbour j of i lies in
// a group g with |c_i - c_g| <= r_i + R_g, since R_g >= |c_j - c_g| + r_j;
// a 1e-6 bohr margin covers rounding), then the candidate groups' members
// with the same overlap test as k_csr.  The fill pass ranks the sphere's
// neighbours (all distinct) into ascending order, so the list is the one
// k_csr writes.  Neighbour counts are at most 255 (checked before the fill).
template <bool FILL>
__global__ void __launch_bounds__(256) k_csr_cells(int nsph, const double4* __restrict__ sph,
                                                   const ZGroups zg, int* cnt, const int* inl,
                                                   int* nl) {
  __shared__ int buf[8][256];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * 8 + w;
  if (i >= nsph) return;  // warp-uniform; no block barriers
  const double4 ci = sph[i];
  int found = 0;
  for (int g0 = 0; g0 < zg.ngroup; g0 += 32) {
    const int g = g0 + lane;
    bool cand = false;
    if (g < zg.ngroup) {
      const double4 cg = zg.gcen[g];
      const double dx = ci.x - cg.x, dy = ci.y - cg.y, dz = ci.z - cg.z;
      const double lim = ci.w + cg.w + 1e-6;
      cand = dx * dx + dy * dy + dz * dz <= lim * lim;
    }
    unsigned m = __ballot_sync(0xffffffffu, cand);
    while (m) {
      const int gg = g0 + __ffs(m) - 1;
      m &= m - 1;
      const int s0 = zg.gstart[gg], s1 = zg.gstart[gg + 1];
      for (int k0 = s0; k0 < s1; k0 += 32) {
        const int k = k0 + lane;
        int j = -1;
        bool nb = false;
        if (k < s1) {
          j = zg.gsph[k];
          nb = j != i && is_nb(ci, sph[j]);
        }
        const unsigned bm = __ballot_sync(0xffffffffu, nb);
        if (FILL && nb) {
          const int pos = found + __popc(bm & ((1u << lane) - 1u));
          if (pos < 256) buf[w][pos] = j;
        }
        found += __popc(bm);
      }
    }
  }
  if constexpr (!FILL) {
    if (lane == 0) cnt[i] = found;
  } else {
    __syncwarp();
    const int base = inl[i], nf = min(found, 256);
    for (int e = lane; e < nf; e += 32) {
      const int v = buf[w][e];
      int r = 0;
      for (int f = 0; f < nf; ++f) r += buf[w][f] < v;
      nl[base + r] = v;
    }
  }
}
cudaError_t launch_csr_count_cells(Launch L, int nsph, const double4* sph, const ZGroups& zg,
                                   int* cnt) {
  k_csr_cells<false><<<(nsph + 7) / 8, 256, 0, L.st>>>(nsph, sph, zg, cnt, nullptr, nullptr);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_csr_fill_cells(Launch L, int nsph, const double4* sph, const ZGroups& zg,
                                  const int* inl, int* nl) {
  k_csr_cells<true><<<(nsph + 7) / 8, 256, 0, L.st>>>(nsph, sph, zg, nullptr, inl, nl);
  ++*L.launches;
  return cudaGetLastError();
}

// rev[k] for k = (i, j): position of i in the neighbour list of j
__global__ void k_csr_rev(int nsph, const int* __restrict__ inl, const int* __restrict__ nl,
                          int* rev) {
  int i = blockIdx.x;
  for (int k = inl[i] + threadIdx.x; k < inl[i + 1]; k += blockDim.x) {
    int j = nl[k];
    int lo = inl[j], hi = inl[j + 1] - 1, pos = -1;
    while (lo <= hi) {
      int mid = (lo + hi) >> 1;
      int v = nl[mid];
      if (v == i) { pos = mid; break; }
      if (v < i) lo = mid + 1; else hi = mid - 1;
    }
    rev[k] = pos;
  }
}
cudaError_t launch_csr_rev(Launch L, int nsph, const int* inl, const int* nl, int* rev) {
  if (nsph == 0) return cudaSuccess;
  k_csr_rev<<<nsph, 32, 0, L.st>>>(nsph, inl, nl, rev);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// fi, ui, zi (ddcosmo.f90:363-411) and the per-point count of containing
// neighbours.  Thread per (sphere, grid point); a sphere's points are taken
// in patch order, padded to whole warps, so that a warp's 32 points lie
// close together on the sphere and skip together the neighbours whose cap
// they all miss (rel_outside: those add exactly nothing).  Each point sums
// its neighbours in CSR order, as the reference does.
// ---------------------------------------------------------------------------
__global__ void k_fiui(const YlmTables tb, int nsph, const double4* __restrict__ sph,
                       const double4* __restrict__ grid, const int* __restrict__ gord,
                       const int* __restrict__ inl, const int* __restrict__ nl, double* fi,
                       double* ui, double* zi, uint8_t* ntri) {
  const int G = tb.ngrid, GP = (G + 31) & ~31;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nsph * GP) return;
  const int i = (int)(t / GP), slot = (int)(t - (long long)i * GP);
  if (slot >= G) return;
  const int n = gord[slot];
  const long long p = (long long)i * G + n;
  double4 ci = sph[i], g = grid[n];
  double f = 0.0, zx = 0.0, zy = 0.0, zz = 0.0;
  int cnt = 0;
  const double eta = tb.eta;
  for (int k = inl[i]; k < inl[i + 1]; k++) {
    double4 cj = sph[nl[k]];
    if (rel_outside(ci, g, cj)) continue;  // t >= 1: no contribution
    Rel r = rel_exact(ci, g, cj);
    double xt = fsw_exact(r.t, eta);
    if (zi && r.t < 1.0 && r.t > DSUB(1.0, eta)) {
      double fac = DDIV(dfsw_exact(r.t, eta), cj.w);
      zx = DADD(zx, DDIV(DMUL(fac, r.vx), r.vv));
      zy = DADD(zy, DDIV(DMUL(fac, r.vy), r.vv));
      zz = DADD(zz, DDIV(DMUL(fac, r.vz), r.vv));
    }
    f = DADD(f, xt);
    if (r.t < 1.0) cnt++;
  }
  fi[p] = f;
  ui[p] = f <= 1.0 ? DSUB(1.0, f) : 0.0;
  ntri[p] = (uint8_t)(cnt > 255 ? 255 : cnt);
  if (zi) {
    zi[3 * p + 0] = zx;
    zi[3 * p + 1] = zy;
    zi[3 * p + 2] = zz;
  }
}
cudaError_t launch_fiui(Launch L, const YlmTables& tb, int nsph, const double4* sph,
                        const double4* grid, const int* gord, const int* inl, const int* nl,
                        double* fi, double* ui, double* zi, uint8_t* ntri) {
  const long long nt = (long long)nsph * ((tb.ngrid + 31) & ~31);
  if (nt == 0) return cudaSuccess;
  k_fiui<<<(unsigned)((nt + 255) / 256), 256, 0, L.st>>>(tb, nsph, sph, grid, gord, inl, nl, fi,
                                                         ui, zi, ntri);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// cavity compaction (ddcosmo.f90:422-468): points with ui > 0, sphere-major
// ---------------------------------------------------------------------------
__global__ void k_cav_count(int ngrid, const double* __restrict__ ui, int* cnt) {
  int i = blockIdx.x;
  int c = 0;
  for (int n = threadIdx.x; n < ngrid; n += blockDim.x) c += ui[(size_t)i * ngrid + n] > 0.0;
  typedef cub::BlockReduce<int, 256> BR;
  __shared__ typename BR::TempStorage tmp;
  int tot = BR(tmp).Sum(c);
  if (threadIdx.x == 0) cnt[i] = tot;
}
cudaError_t launch_cav_count(Launch L, int nsph, int ngrid, const double* ui, int* cnt) {
  if (nsph == 0) return cudaSuccess;
  k_cav_count<<<nsph, 256, 0, L.st>>>(ngrid, ui, cnt);
  ++*L.launches;
  return cudaGetLastError();
}

__global__ void k_cav_fill(int ngrid, const double* __restrict__ ui,
                           const double4* __restrict__ sph, const double4* __restrict__ grid,
                           const int* __restrict__ cavoff, int* cavidx, int* cavpt, double* ccav) {
  int i = blockIdx.x;
  typedef cub::BlockScan<int, 256> BS;
  __shared__ typename BS::TempStorage tmp;
  __shared__ int carry;
  if (threadIdx.x == 0) carry = cavoff[i];
  __syncthreads();
  double4 ci = sph[i];
  for (int n0 = 0; n0 < ngrid; n0 += 256) {
    int n = n0 + threadIdx.x;
    size_t p = (size_t)i * ngrid + n;
    int flag = (n < ngrid && ui[p] > 0.0) ? 1 : 0;
    int pos, tot;
    BS(tmp).ExclusiveSum(flag, pos, tot);
    int base = carry;
    if (n < ngrid) {
      if (flag) {
        int c = base + pos;
        double4 g = grid[n];
        cavidx[p] = c;
        cavpt[c] = (int)p;
        ccav[3 * (size_t)c + 0] = DADD(ci.x, DMUL(ci.w, g.x));
        ccav[3 * (size_t)c + 1] = DADD(ci.y, DMUL(ci.w, g.y));
        ccav[3 * (size_t)c + 2] = DADD(ci.z, DMUL(ci.w, g.z));
      } else {
        cavidx[p] = -1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) carry = base + tot;
    __syncthreads();
  }
}
cudaError_t launch_cav_fill(Launch L, int nsph, int ngrid, const double* ui, const double4* sph,
                            const double4* grid, const int* cavoff, int* cavidx, int* cavpt,
                            double* ccav) {
  if (nsph == 0) return cudaSuccess;
  k_cav_fill<<<nsph, 256, 0, L.st>>>(ngrid, ui, sph, grid, cavoff, cavidx, cavpt, ccav);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// pair-major triple lists: for CSR entry k = (i, j), the grid points n of
// sphere i with t_n^ij < 1 (calcv's test, ddcosmo.f90:1707-1716).  Warp per
// pair, ballot over points in ascending order.
// ---------------------------------------------------------------------------
// The count pass stores each pair's membership bits (one 32-bit word per 32
// grid points), and the fill pass expands them: the exact geometry of every
// (pair, point) is evaluated once
template <bool FILL>
__global__ void k_pairs(int nsph, int npair, int ngrid, const double4* __restrict__ sph,
                        const double4* __restrict__ grid, const int* __restrict__ inl,
                        const int* __restrict__ nl, int* cnt, unsigned* __restrict__ bits,
                        const int* pn_ptr, uint16_t* pn, uint8_t* pn_pair) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= npair) return;
  const int k = warp;
  const int nw = (ngrid + 31) >> 5;
  unsigned* kb = bits + (size_t)k * nw;
  if constexpr (!FILL) {
    // sphere owning entry k: binary search in inl
    int lo = 0, hi = nsph - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (inl[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const int i = lo, j = nl[k];
    const double4 ci = sph[i], cj = sph[j];
    int total = 0;
    for (int w = 0; w < nw; ++w) {
      const int n = 32 * w + lane;
      bool in = false;
      if (n < ngrid) in = rel_exact(ci, grid[n], cj).t < 1.0;
      const unsigned mask = __ballot_sync(0xffffffffu, in);
      if (lane == 0) kb[w] = mask;
      total += __popc(mask);
    }
    if (lane == 0) cnt[k] = total;
  } else {
    int lo = 0, hi = nsph - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (inl[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const int i = lo;
    int base = pn_ptr[k];
    for (int w = 0; w < nw; ++w) {
      const unsigned mask = kb[w];
      if ((mask >> lane) & 1u) {
        const int pos = base + __popc(mask & ((1u << lane) - 1u));
        pn[pos] = (uint16_t)(32 * w + lane);
        pn_pair[pos] = (uint8_t)(k - inl[i]);
      }
      base += __popc(mask);
    }
  }
}
cudaError_t launch_pair_count(Launch L, int nsph, int npair, int ngrid, const double4* sph,
                              const double4* grid, const int* inl, const int* nl, int* cnt,
                              unsigned* bits) {
  if (npair == 0) return cudaSuccess;
  k_pairs<false><<<(npair + 7) / 8, 256, 0, L.st>>>(nsph, npair, ngrid, sph, grid, inl, nl, cnt,
                                                    bits, nullptr, nullptr, nullptr);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_pair_fill(Launch L, int nsph, int npair, int ngrid, const double4* sph,
                             const double4* grid, const int* inl, const int* nl,
                             const unsigned* bits, const int* pn_ptr, uint16_t* pn,
                             uint8_t* pn_pair) {
  if (npair == 0) return cudaSuccess;
  k_pairs<true><<<(npair + 7) / 8, 256, 0, L.st>>>(nsph, npair, ngrid, sph, grid, inl, nl,
                                                   nullptr, const_cast<unsigned*>(bits), pn_ptr,
                                                   pn, pn_pair);
  ++*L.launches;
  return cudaGetLastError();
}

// adjoint gather list: for sphere i, for j in N_i (CSR order), points of j
// inside i = pair list of entry rev(k) (adjrhs ddcosmo.f90:1316-1381)
__global__ void k_ls_count(int nsph, const int* __restrict__ inl, const int* __restrict__ rev,
                           const int* __restrict__ pn_ptr, int* cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsph) return;
  int c = 0;
  for (int k = inl[i]; k < inl[i + 1]; k++) {
    int kk = rev[k];
    c += pn_ptr[kk + 1] - pn_ptr[kk];
  }
  cnt[i] = c;
}
cudaError_t launch_ls_count(Launch L, int nsph, const int* inl, const int* rev, const int* pn_ptr,
                            int* cnt) {
  if (nsph == 0) return cudaSuccess;
  k_ls_count<<<(nsph + 127) / 128, 128, 0, L.st>>>(nsph, inl, rev, pn_ptr, cnt);
  ++*L.launches;
  return cudaGetLastError();
}
__global__ void k_ls_fill(int nsph, const int* __restrict__ inl, const int* __restrict__ nl,
                          const int* __restrict__ rev, const int* __restrict__ pn_ptr,
                          const uint16_t* __restrict__ pn, const int* __restrict__ ls_ptr,
                          int2* ls, int* lsstart) {
  int i = blockIdx.x;
  int off = ls_ptr[i];
  for (int k = inl[i]; k < inl[i + 1]; k++) {
    int kk = rev[k], j = nl[k];
    int a = pn_ptr[kk], b = pn_ptr[kk + 1];
    if (threadIdx.x == 0) lsstart[kk] = off;  // where pair (j, i) sits in i's gather list
    for (int q = a + threadIdx.x; q < b; q += blockDim.x) ls[off + (q - a)] = make_int2(j, pn[q]);
    off += b - a;
  }
}
cudaError_t launch_ls_fill(Launch L, int nsph, const int* inl, const int* nl, const int* rev,
                           const int* pn_ptr, const uint16_t* pn, const int* ls_ptr, int2* ls,
                           int* lsstart) {
  if (nsph == 0) return cudaSuccess;
  k_ls_fill<<<nsph, 128, 0, L.st>>>(nsph, inl, nl, rev, pn_ptr, pn, ls_ptr, ls, lsstart);
  ++*L.launches;
  return cudaGetLastError();
}

__global__ void k_sum_counts(const int* __restrict__ cnt, int n, unsigned long long* out) {
  unsigned long long v = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v += (unsigned long long)(unsigned)cnt[i];
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(out, v);  // integer sum: order-free
}
cudaError_t launch_sum_counts(Launch L, const int* cnt, int n, unsigned long long* out) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), L.st);
  if (e || n <= 0) return e;
  k_sum_counts<<<std::min((n + 255) / 256, 148 * 4), 256, 0, L.st>>>(cnt, n, out);
  ++*L.launches;
  return cudaGetLastError();
}

size_t scan_temp_bytes(int n) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const int*)nullptr, (int*)nullptr, n + 1);
  return b;
}
// in[0..n-1] -> out[0..n] with out[n] = total (in[n] must be readable: the
// caller passes n+1 entries with in[n] = 0)
cudaError_t scan_exclusive(Launch L, const int* in, int* out, int n, void* temp,
                           size_t temp_bytes) {
  return cub::DeviceScan::ExclusiveSum(temp, temp_bytes, in, out, n + 1, L.st);
}

// ---------------------------------------------------------------------------
// Spherical-harmonic contraction for the matvecs.  m-outer / l-inner
// Legendre recurrence (polleg, ddcosmo.f90:1056-1094) with t^l folded in:
//   Pt_l^m = t^l P_l^m,  Pt_m^m = t^m P_m^m,
//   Pt_{m+1}^m = (2m+1) c t Pt_m^m,  Pt_l^m = A c t Pt_{l-1}^m - B t^2 Pt_{l-2}^m
// cos(m phi), sin(m phi) by the Chebyshev recurrence (trgev :1103-1125).
// ---------------------------------------------------------------------------
struct Angles {
  double c, s, cp, sp;  // cos/sin theta, cos/sin phi
};
__device__ __forceinline__ Angles angles_of(double sx, double sy, double sz) {
  Angles a;
  a.c = sz;
  a.s = sqrt(fmax(0.0, 1.0 - sz * sz));
  if (a.s != 0.0) {
    double r = 1.0 / a.s;
    a.cp = sx * r;
    a.sp = sy * r;
  } else {  // pole: only m = 0 survives (P_l^m = 0 for m > 0)
    a.cp = 1.0;
    a.sp = 0.0;
  }
  return a;
}

// X of one sphere staged as pairs (X_{l,m}, X_{l,-m}) * K_lm, index lmi(l,m)
template <int LMAX>
__device__ __forceinline__ double ylm_dot(const YlmTables& tb, const Angles& a, double t,
                                          const double2* __restrict__ xs) {
  const double ct = a.c * t, st = a.s * t, t2 = t * t;
  double acc = 0.0;
  double pmm = 1.0;                     // Pt_m^m
  double cm = 1.0, sm = 0.0, cmm1 = 1.0, smm1 = 0.0;
#pragma unroll
  for (int m = 0; m <= LMAX; ++m) {
    if (m == 1) {
      cm = a.cp;
      sm = a.sp;
    } else if (m >= 2) {
      double cn = 2.0 * a.cp * cm - cmm1, sn = 2.0 * a.cp * sm - smm1;
      cmm1 = cm; smm1 = sm; cm = cn; sm = sn;
    }
    double p0 = pmm, p1 = 0.0;
#pragma unroll
    for (int l = m; l <= LMAX; ++l) {
      double P;
      if (l == m) {
        P = p0;
      } else if (l == m + 1) {
        p1 = (2.0 * m + 1.0) * ct * p0;
        P = p1;
      } else {
        P = (tb.A[lmi(l, m)] * ct) * p1 - (tb.B[lmi(l, m)] * t2) * p0;
        p0 = p1;
        p1 = P;
      }
      double2 xv = xs[lmi(l, m)];
      double q = (m == 0) ? xv.x : fma(cm, xv.x, sm * xv.y);
      acc = fma(P, q, acc);
    }
    pmm = -pmm * (2.0 * m + 1.0) * st;
  }
  return acc;
}

// ---------------------------------------------------------------------------
// lx, part 1 (calcv ddcosmo.f90:1671-1746 with intmlp :1140-1178), second
// form, both precisions.  Block per sphere i:
//   * K*X_j of every neighbour j (as (X_{l,m}, X_{l,-m}) pairs) and the
//     centre differences c_i - c_j are staged in shared memory once;
//   * the sphere's triples (pair-major list) are spread over all threads, a
//     per-triple local pair index selects the staged neighbour;
//   * contributions to the same grid point inside one warp instruction are
//     combined in lane order (match_any) before the warp-private row update,
//     so the sum order is fixed and the result bit-reproducible;
//   * one accumulator per m column keeps independent FMA chains in flight.
// ---------------------------------------------------------------------------
template <class Rl> struct RT;
template <> struct RT<double> {
  typedef double2 V2;
};
template <> struct RT<float> {
  typedef float2 V2;
};
template <class Rl> __device__ __forceinline__ typename RT<Rl>::V2 mk2(Rl a, Rl b);
template <> __device__ __forceinline__ double2 mk2<double>(double a, double b) {
  return make_double2(a, b);
}
template <> __device__ __forceinline__ float2 mk2<float>(float a, float b) {
  return make_float2(a, b);
}
template <class Rl> struct GP {
  Rl x, y, z, w;
};
__device__ __forceinline__ GP<double> grid_pt(const DevGeo& g, int n, double*) {
  double4 v = g.grid[n];
  return GP<double>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ GP<float> grid_pt(const DevGeo& g, int n, float*) {
  float4 v = g.gridf[n];
  return GP<float>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
// 1/sqrt(x) for a positive normal x (a squared distance between distinct
// points) in the N-body sums: the hardware estimate rsqrt.approx.ftz.f64,
// then one third-order Householder step y (1 + h/2 + 3h^2/8), h = 1 - x y^2
// (the binomial series of (1 - h)^(-1/2) to second order).  The step cubes
// the estimate's relative error, so the result carries only the rounding of
// its five FP64 operations; no special-value handling is needed for such x.
__device__ __forceinline__ double rsqrt_pos(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double h = fma(-x, y * y, 1.0);
  return fma(y * h, fma(h, 0.375, 0.5), y);
}
__device__ __forceinline__ double sqrt_t(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_t(float x) { return sqrtf(x); }

// K-scaled copy of X in (X_{l,m}, X_{l,-m}) pair layout, [N][NLM]
template <class Rl, bool GAM = false>
__global__ void k_xk(const YlmTables tb, int nsph, const double* __restrict__ X,
                     typename RT<Rl>::V2* XK) {
  const int nlm = (tb.lmax + 1) * (tb.lmax + 2) / 2;
  // 32-bit indices (nsph * nlm < 2^31, checked at launch)
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsph * nlm) return;
  const int i = e / nlm, le = e - i * nlm;
  int l = 0;
  while (lmi(l + 1, 0) <= le) ++l;
  const int m = le - lmi(l, 0), ind = l * l + l;
  const double* Xi = X + (size_t)i * tb.nylm;
  const double kk = GAM ? tb.Kg[le] : tb.K[le];
  XK[e] = mk2<Rl>((Rl)(kk * Xi[ind + m]), m ? (Rl)(kk * Xi[ind - m]) : Rl(0));
}

#define DDC_LMAX_CASES(X) \
  X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)

// ---------------------------------------------------------------------------
// lstarx (adjrhs ddcosmo.f90:1301-1384, matvec.f90:161-235):
//   y_i,lm = - sum_{j in N_i} sum_{n: t_n^ji<1} w_n xi_j(n) W_ji(n)
//                4pi/(2l+1) t^l Y_lm(s_n^ji)
// Block per sphere i, one warp per "role".  A role owns the Legendre
// columns m and lmax-m (and the middle column when lmax is even), which
// balances the recurrence work (lmax+2 steps per role) and caps the
// register accumulators at 2*lmax+4.  Per chunk of triples (one per thread):
//   phase A: every thread computes one triple's geometry, weight and the
//            prefix Pt_m^m (coef folded in), cos(m phi), sin(m phi) for all m
//            into shared memory;
//   phase B: each role warp runs its columns over the chunk, lanes over
//            triples, accumulating in registers.
// At the end each role reduces its accumulators across its 32 lanes with a
// fixed shuffle tree.  No atomics: the result is bit-reproducible.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ls_nroles(int L) { return L / 2 + 1; }
__host__ __device__ constexpr int ls_col2(int L, int r) { return L - r; }  // second column
__host__ __device__ constexpr bool ls_has2(int L, int r) { return L - r > r; }
__host__ __device__ constexpr int ls_nvals_m(int L, int m) { return m == 0 ? L + 1 : 2 * (L + 1 - m); }
__host__ __device__ constexpr int ls_role_nvals(int L, int r) {
  return ls_nvals_m(L, r) + (ls_has2(L, r) ? ls_nvals_m(L, L - r) : 0);
}
// shared-memory fields per triple: ct, t2, then pmm[m], cos[m], sin[m]
__host__ __device__ constexpr int ls_nfields(int L) { return 2 + 3 * (L + 1); }

template <int LMAX, int M, int OFF, class Rl>
__device__ __forceinline__ void ls_column(const YlmTables& tb, Rl ct, Rl t2, Rl p0, Rl cm, Rl sm,
                                          Rl* acc) {
  Rl p1 = 0;
#pragma unroll
  for (int l = M; l <= LMAX; ++l) {
    Rl P;
    if (l == M) {
      P = p0;
    } else if (l == M + 1) {
      p1 = (Rl)(2 * M + 1) * ct * p0;
      P = p1;
    } else {
      P = (cA<Rl>(tb, lmi(l, M)) * ct) * p1 - (cB<Rl>(tb, lmi(l, M)) * t2) * p0;
      p0 = p1;
      p1 = P;
    }
    if (M == 0) {
      acc[OFF + (l - M)] += P;
    } else {
      acc[OFF + (l - M)] = fma(P, cm, acc[OFF + (l - M)]);
      acc[OFF + (LMAX + 1 - M) + (l - M)] = fma(P, sm, acc[OFF + (LMAX + 1 - M) + (l - M)]);
    }
  }
}

// GAM: accumulators of the normalised recurrence (scale Kg instead of K)
template <int LMAX, int M, int OFF, class Rl, bool GAM = false>
__device__ __forceinline__ void ls_store(const YlmTables& tb, const Rl* acc, double* yi,
                                         int lane) {
#pragma unroll
  for (int l = M; l <= LMAX; ++l) {
    const int ind = l * l + l;
    const double k = GAM ? tb.Kg[lmi(l, M)] : tb.K[lmi(l, M)];
    if (M == 0) {
      if (lane == 0) yi[ind] = -k * (double)acc[OFF + (l - M)];
    } else if (lane == 0) {
      yi[ind + M] = -k * (double)acc[OFF + (l - M)];
      yi[ind - M] = -k * (double)acc[OFF + (LMAX + 1 - M) + (l - M)];
    }
  }
}

// fields are stored [field][stride]; lanes take triples q < count
template <int LMAX, int R, class Rl>
__device__ __forceinline__ void ls_role(const YlmTables& tb, const Rl* sh, int stride,
                                        int count, int lane, Rl* acc) {
  constexpr int M1 = R, M2 = LMAX - R;
  for (int q = lane; q < count; q += 32) {
    const Rl ct = sh[q], t2 = sh[stride + q];
    ls_column<LMAX, M1, 0, Rl>(tb, ct, t2, sh[(2 + 3 * M1) * stride + q],
                               sh[(3 + 3 * M1) * stride + q], sh[(4 + 3 * M1) * stride + q], acc);
    if constexpr (ls_has2(LMAX, R))
      ls_column<LMAX, M2, ls_nvals_m(LMAX, M1), Rl>(tb, ct, t2, sh[(2 + 3 * M2) * stride + q],
                                                     sh[(3 + 3 * M2) * stride + q],
                                                     sh[(4 + 3 * M2) * stride + q], acc);
  }
}

template <int LMAX, int R, class Rl, bool GAM = false>
__device__ __forceinline__ void ls_role_finish(const YlmTables& tb, Rl* acc, double* yi,
                                               int lane) {
  constexpr int NV = ls_role_nvals(LMAX, R);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
  }
  ls_store<LMAX, R, 0, Rl, GAM>(tb, acc, yi, lane);
  if constexpr (ls_has2(LMAX, R))
    ls_store<LMAX, LMAX - R, ls_nvals_m(LMAX, R), Rl, GAM>(tb, acc, yi, lane);
}

// dispatch a runtime role index to the compile-time role code
template <int LMAX, int R, class Rl>
__device__ __forceinline__ void ls_run_role(int role, const YlmTables& tb, const Rl* sh,
                                            int stride, int count, int lane, Rl* acc) {
  if (role == R) {
    ls_role<LMAX, R, Rl>(tb, sh, stride, count, lane, acc);
    return;
  }
  if constexpr (R + 1 < ls_nroles(LMAX))
    ls_run_role<LMAX, R + 1, Rl>(role, tb, sh, stride, count, lane, acc);
}
template <int LMAX, int R, class Rl, bool GAM = false>
__device__ __forceinline__ void ls_finish_role(int role, const YlmTables& tb, Rl* acc,
                                               double* yi, int lane) {
  if (role == R) {
    ls_role_finish<LMAX, R, Rl, GAM>(tb, acc, yi, lane);
    return;
  }
  if constexpr (R + 1 < ls_nroles(LMAX))
    ls_finish_role<LMAX, R + 1, Rl, GAM>(role, tb, acc, yi, lane);
}

__host__ __device__ constexpr int ls_max_nvals(int L) {
  int mx = 0;
  for (int r = 0; r < ls_nroles(L); ++r) mx = ls_role_nvals(L, r) > mx ? ls_role_nvals(L, r) : mx;
  return mx;
}

template <int LMAX>
__global__ void __launch_bounds__(32 * ls_nroles(LMAX)) k_lstarx(const YlmTables tb,
                                                                  const DevGeo g,
                                                                  const double* __restrict__ xi,
                                                                  double* y) {
  constexpr int NR = ls_nroles(LMAX);
  constexpr int NT = 32 * NR;  // threads per block
  constexpr int CH = NT;       // triples per chunk (one per thread in phase A)
  constexpr int NF = ls_nfields(LMAX);
  constexpr int NVM = ls_max_nvals(LMAX);
  extern __shared__ double sh[];  // [NF][CH]
  const int i = blockIdx.x;
  if (sweep_skip(g.act, i)) return;
  const int role = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double4 ci = g.sph[i];
  const int G = g.ngrid;
  const double eta = tb.eta, flow = 1.0 - eta;
  const double fa = 15.0 * eta - 12.0, fb = 10.0 * eta * eta - 15.0 * eta + 6.0;
  const double ie5 = 1.0 / (eta * eta * eta * eta * eta);
  const double iri = 1.0 / ci.w;
  double acc[NVM];
#pragma unroll
  for (int v = 0; v < NVM; ++v) acc[v] = 0.0;
  const int q0 = g.ls_ptr[i], q1 = g.ls_ptr[i + 1];
  for (int c0 = q0; c0 < q1; c0 += CH) {
    const int chunk = min(CH, q1 - c0);
    // phase A: one triple per thread
    for (int tt = threadIdx.x; tt < chunk; tt += NT) {
      const int q = c0 + tt;
      const int2 jn = g.ls[q];
      const int j = jn.x, n = jn.y;
      const double4 cj = g.sph[j];
      const double4 gn = g.grid[n];
      double vx = fma(cj.w, gn.x, cj.x) - ci.x;
      double vy = fma(cj.w, gn.y, cj.y) - ci.y;
      double vz = fma(cj.w, gn.z, cj.z) - ci.z;
      double r2 = vx * vx + vy * vy + vz * vz;
      double rinv = rsqrt(r2);
      double t = r2 * rinv * iri;
      Angles a = angles_of(vx * rinv, vy * rinv, vz * rinv);
      const size_t pj = (size_t)j * G + n;
      double chi = fsw_fast(t, eta, flow, fa, fb, ie5);
      double f = g.fi[pj];
      double W = f > 1.0 ? chi / f : chi;
      const double st = a.s * t;
      double* col = sh + tt;
      col[0] = a.c * t;
      col[CH] = t * t;
      double pmm = gn.w * xi[pj] * W;
      double cm = 1.0, sm = 0.0, cmm1 = 1.0, smm1 = 0.0;
#pragma unroll
      for (int m = 0; m <= LMAX; ++m) {
        if (m == 1) {
          cm = a.cp; sm = a.sp;
        } else if (m >= 2) {
          double cn = 2.0 * a.cp * cm - cmm1, sn = 2.0 * a.cp * sm - smm1;
          cmm1 = cm; smm1 = sm; cm = cn; sm = sn;
        }
        col[(2 + 3 * m) * CH] = pmm;
        col[(3 + 3 * m) * CH] = cm;
        col[(4 + 3 * m) * CH] = sm;
        pmm = -pmm * (2.0 * m + 1.0) * st;
      }
    }
    __syncthreads();
    // phase B: the role's columns over the chunk
    ls_run_role<LMAX, 0, double>(role, tb, sh, CH, chunk, lane, acc);
    __syncthreads();
  }
  ls_finish_role<LMAX, 0, double>(role, tb, acc, y + (size_t)i * tb.nylm, lane);
}

cudaError_t launch_lstarx_acc(Launch L, const YlmTables& tb, const DevGeo& g, const double* xi,
                              double* y) {
  if (g.nsph == 0) return cudaSuccess;
  cudaError_t e = cudaSuccess;
#define CASE(LV)                                                                              \
  case LV: {                                                                                  \
    constexpr int NR = ls_nroles(LV);                                                         \
    size_t sm = sizeof(double) * ls_nfields(LV) * 32 * NR;                                    \
    if (sm > 48 * 1024)                                                                       \
      if ((e = cudaFuncSetAttribute(k_lstarx<LV>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                    (int)sm)))                                                \
        return e;                                                                             \
    k_lstarx<LV><<<g.nsph, 32 * NR, sm, L.st>>>(tb, g, xi, y);                                \
    break;                                                                                    \
  }
  switch (tb.lmax) {
    DDC_LMAX_CASES(CASE)
    default:
      return cudaErrorInvalidValue;
  }
#undef CASE
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Register-tiled SIMT GEMM, column-major C[M x N] = alpha * op(A) * B: the
// FP32 projection and expansion of the mixed path when the harmonics do not
// fit one 128-row tensor-core tile (lmax 11, 12).  BM x BN tile per block,
// BK deep, TM x TN outputs per thread, shared tiles double buffered with the
// next tile prefetched into registers.  Acc is the arithmetic/accumulation
// type; inputs are converted when staged.
// ---------------------------------------------------------------------------
template <bool TA, class TAin, class TBin, class TC, class Acc, int BM, int BN, int BK, int TM,
          int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_gemm2(int M, int N, int K, Acc alpha,
                                                                 const TAin* __restrict__ A,
                                                                 int lda,
                                                                 const TBin* __restrict__ B,
                                                                 int ldb, TC* C, int ldc) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int NA = BM * BK / NT, NB = BK * BN / NT;  // staged elements per thread
  __shared__ __align__(16) Acc As[2][BK][BM];
  __shared__ __align__(16) Acc Bs[2][BK][BN];
  const int tx = threadIdx.x % (BN / TN), ty = threadIdx.x / (BN / TN);
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  Acc ra[NA], rb[NB];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int u = 0; u < NA; ++u) {
      const int e = threadIdx.x + u * NT;
      int mm, kk;
      if (TA) { kk = e % BK; mm = e / BK; } else { mm = e % BM; kk = e / BM; }
      const int m = m0 + mm, k = k0 + kk;
      Acc v = 0;
      if (m < M && k < K) v = (Acc)(TA ? A[(size_t)m * lda + k] : A[(size_t)k * lda + m]);
      ra[u] = v;
    }
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      const int e = threadIdx.x + u * NT;
      const int kk = e % BK, nn = e / BK;
      const int n = n0 + nn, k = k0 + kk;
      rb[u] = (n < N && k < K) ? (Acc)B[(size_t)n * ldb + k] : Acc(0);
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int u = 0; u < NA; ++u) {
      const int e = threadIdx.x + u * NT;
      int mm, kk;
      if (TA) { kk = e % BK; mm = e / BK; } else { mm = e % BM; kk = e / BM; }
      As[buf][kk][mm] = ra[u];
    }
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      const int e = threadIdx.x + u * NT;
      Bs[buf][e % BK][e / BK] = rb[u];
    }
  };
  Acc acc[TM][TN];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TN; ++b) acc[a][b] = 0;
  fetch(0);
  stash(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += BK) {
    const bool more = k0 + BK < K;
    if (more) fetch(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      Acc a[TM], b[TN];
#pragma unroll
      for (int r = 0; r < TM; ++r) a[r] = As[buf][kk][ty * TM + r];
#pragma unroll
      for (int c = 0; c < TN; ++c) b[c] = Bs[buf][kk][tx * TN + c];
#pragma unroll
      for (int r = 0; r < TM; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    if (more) {
      stash(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
#pragma unroll
  for (int r = 0; r < TM; ++r)
#pragma unroll
    for (int c = 0; c < TN; ++c) {
      const int m = m0 + ty * TM + r, n = n0 + tx * TN + c;
      if (m < M && n < N) C[(size_t)n * ldc + m] = (TC)(alpha * acc[r][c]);
    }
}

template <bool TA, class TAin, class TBin, class TC, class Acc>
cudaError_t gemm2(Launch L, int M, int N, int K, Acc alpha, const TAin* A, int lda, const TBin* B,
                  int ldb, TC* C, int ldc) {
  if (M == 0 || N == 0) return cudaSuccess;
  // FP32: 128x64 tiles, 8x4 per thread; FP64: 128x32 tiles, 8x2 per thread
  constexpr bool D = sizeof(Acc) == 8;
  constexpr int BM = 128, BN = D ? 32 : 64, TM = 8, TN = D ? 2 : 4, BK = D ? 8 : 16;
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
  k_gemm2<TA, TAin, TBin, TC, Acc, BM, BN, BK, TM, TN>
      <<<grid, (BM / TM) * (BN / TN), 0, L.st>>>(M, N, K, alpha, A, lda, B, ldb, C, ldc);
  ++*L.launches;
  return cudaGetLastError();
}

// FP64 GEMM of the operators' projection and expansion (FP64 path, the
// refinement steps and the one-off RHS projections) on the FP64 tensor
// cores (DMMA, mma.sync m8n8k4; tcgen05 has no FP64 kind):
//   C[n*ldc + m] = alpha * sum_k A[k*lda + m] B[n*ldb + k].
// 128 x 64 tiles, 8 warps of 32 x 32 (4 x 4 MMA tiles of 8 x 8), 16-deep k
// slabs copied to shared memory with cp.async (the next slab in flight).
// Shared rows are padded so that each warp's fragment loads take the
// minimum two wavefronts: A rows of 136 doubles (a row stride of 16 banks
// mod 32 separates k and k + 1), B rows of 20 (8 banks mod 32 separates
// four columns).  Each output is one FMA chain in k order.
namespace dgp {
constexpr int BM = 128, BN = 64, BK = 16;
constexpr int AS = BM + 8, BS = BK + 4;
constexpr int SMEM = (2 * BK * AS + 2 * BN * BS) * 8;
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc, bool valid) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  const int n = valid ? 8 : 0;  // 0: nothing read, the destination is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(gsrc), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__global__ void __launch_bounds__(256, 3) k_dgemm_dmma(int M, int N, int K, double alpha,
                                                       const double* __restrict__ A, int lda,
                                                       const double* __restrict__ B, int ldb,
                                                       double* __restrict__ C, int ldc,
                                                       const SweepMask act) {
  using namespace dgp;
  extern __shared__ __align__(16) double dg_smem[];
  double* As = dg_smem;                // [2][BK][AS]
  double* Bs = dg_smem + 2 * BK * AS;  // [2][BN][BS]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp & 3, wn = warp >> 2;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  // columns are spheres: a batched sweep skips a tile whose spheres all belong
  // to stopped molecules
  if (act.mol && __syncthreads_and(tid >= BN || n0 + tid >= N || sweep_skip(act, n0 + tid)))
    return;
  auto load = [&](int buf, int k0) {
#pragma unroll
    for (int u = 0; u < BM * BK / 256; ++u) {
      const int e = tid + u * 256;
      const int mm = e % BM, kk = e / BM;
      const int m = m0 + mm, k = k0 + kk;
      const bool ok = m < M && k < K;
      cp_async8(As + (buf * BK + kk) * AS + mm, ok ? A + (size_t)k * lda + m : A, ok);
    }
#pragma unroll
    for (int u = 0; u < BN * BK / 256; ++u) {
      const int e = tid + u * 256;
      const int kk = e % BK, nn = e / BK;
      const int n = n0 + nn, k = k0 + kk;
      const bool ok = n < N && k < K;
      cp_async8(Bs + (buf * BN + nn) * BS + kk, ok ? B + (size_t)n * ldb + k : B, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nk = (K + BK - 1) / BK;
  const int fr = lane >> 2, fk = lane & 3;  // fragment row / k of this lane
  load(0, 0);
  for (int t = 0; t < nk; ++t) {
    const int buf = t & 1;
    if (t + 1 < nk) {
      load(buf ^ 1, (t + 1) * BK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const double* as = As + buf * BK * AS;
    const double* bs = Bs + buf * BN * BS;
#pragma unroll
    for (int ks = 0; ks < BK; ks += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[(ks + fk) * AS + wm * 32 + i * 8 + fr];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[(wn * 32 + j * 8 + fr) * BS + ks + fk];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          asm volatile(
              "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
              : "+d"(acc[i][j][0]), "+d"(acc[i][j][1])
              : "d"(a[i]), "d"(b[j]));
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = m0 + wm * 32 + i * 8 + fr;
        const int n = n0 + wn * 32 + j * 8 + 2 * fk + h;
        if (m < M && n < N) C[(size_t)n * ldc + m] = alpha * acc[i][j][h];
      }
}
// dst[c*rows + r] = src[r*cols + c]
__global__ void k_transpose(int rows, int cols, const double* __restrict__ src, double* dst) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)rows * cols) return;
  const int r = (int)(e / cols), c = (int)(e - (long long)r * cols);
  dst[(size_t)c * rows + r] = src[e];
}
cudaError_t launch_transpose(Launch L, int rows, int cols, const double* src, double* dst) {
  const long long n = (long long)rows * cols;
  if (n == 0) return cudaSuccess;
  k_transpose<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(rows, cols, src, dst);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_dgemm_nn(Launch L, int M, int N, int K, double alpha, const double* A,
                            int lda, const double* B, int ldb, double* C, int ldc,
                            const SweepMask& act) {
  if (M == 0 || N == 0) return cudaSuccess;
  dim3 grid((M + dgp::BM - 1) / dgp::BM, (N + dgp::BN - 1) / dgp::BN);
  cudaError_t e = cudaFuncSetAttribute(k_dgemm_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       dgp::SMEM);
  if (e) return e;
  k_dgemm_dmma<<<grid, 256, dgp::SMEM, L.st>>>(M, N, K, alpha, A, lda, B, ldb, C, ldc, act);
  ++*L.launches;
  return cudaGetLastError();
}
// FP32 SIMT contractions of the mixed path where the tensor-core kernels do
// not apply (more than 128 harmonics): projection into FP64 y, and xi of the
// FP64 vector s
cudaError_t launch_proj_f32_simt(Launch L, int nylm, int nsph, int ngrid, float alpha,
                                 const float* bw_f, const float* pot, int ldp, double* y) {
  return gemm2<false, float, float, double, float>(L, nylm, nsph, ngrid, alpha, bw_f, nylm, pot,
                                                   ldp, y, nylm);
}
cudaError_t launch_xi_f32_simt(Launch L, int nylm, int nsph, int ngrid, const float* basis_f,
                               const double* s, float* xi) {
  return gemm2<true, float, double, float, float>(L, ngrid, nsph, nylm, 1.f, basis_f, nylm, s,
                                                  nylm, xi, ngrid);
}


// wghpot (ddcosmo.f90:1187-1224): g(n,i) = -ui * phi(cavity index)
__global__ void k_wghpot(long long np, const double* __restrict__ ui, const int* __restrict__ cavidx,
                         const double* __restrict__ phi, double* gb) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  int c = cavidx[p];
  gb[p] = c >= 0 ? -ui[p] * phi[c] : 0.0;
}
cudaError_t launch_wghpot(Launch L, const DevGeo& g, const double* phi, double* gbuf) {
  long long np = (long long)g.nsph * g.ngrid;
  if (np == 0) return cudaSuccess;
  k_wghpot<<<(unsigned)((np + 255) / 256), 256, 0, L.st>>>(np, g.ui, g.cavidx, phi, gbuf);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// vector kernels of the Jacobi/DIIS solver (jacobi_diis.f90)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int l_of(int lm) {
  int l = (int)sqrtf((float)lm);
  while ((l + 1) * (l + 1) <= lm) ++l;
  while (l * l > lm) --l;
  return l;
}

// Grid-stride walk over the (nylm, nsph) vectors that keeps the harmonic
// index lm = q mod nylm incrementally (no 64-bit division per element).
struct LmWalk {
  long long q, stride;
  int lm, dlm, nylm;
  __device__ LmWalk(int nylm_) : nylm(nylm_) {
    q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    stride = (long long)gridDim.x * blockDim.x;
    lm = (int)(q % nylm);
    dlm = (int)(stride % nylm);
  }
  __device__ void next() {
    q += stride;
    lm += dlm;
    if (lm >= nylm) lm -= nylm;
  }
};

__global__ void k_ldm1x(const YlmTables tb, long long n, const double* __restrict__ x, double* y) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  int lm = (int)(e % tb.nylm);
  y[e] = tb.facl[l_of(lm)] * x[e];
}
cudaError_t launch_ldm1x(Launch L, const YlmTables& tb, long long n, const double* x, double* y) {
  if (n == 0) return cudaSuccess;
  k_ldm1x<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(tb, n, x, y);
  ++*L.launches;
  return cudaGetLastError();
}
__global__ void k_scale(long long n, double a, const double* __restrict__ x, double* y) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) y[e] = a * x[e];
}
cudaError_t launch_scale(Launch L, long long n, double a, const double* x, double* y) {
  if (n == 0) return cudaSuccess;
  k_scale<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(n, a, x, y);
  ++*L.launches;
  return cudaGetLastError();
}
// mode 0: x = facl * rhs (cosmo.f90:136-138), 1: x = 0
__global__ void k_guess(const YlmTables tb, long long n, const double* __restrict__ rhs, double* x,
                        int mode) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  x[e] = mode == 0 ? tb.facl[l_of((int)(e % tb.nylm))] * rhs[e] : 0.0;
}
cudaError_t launch_guess(Launch L, const YlmTables& tb, long long n, const double* rhs, double* x,
                         int mode) {
  if (n == 0) return cudaSuccess;
  k_guess<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(tb, n, rhs, x, mode);
  ++*L.launches;
  return cudaGetLastError();
}

int reduce_blocks() { return 148 * 4; }

// block sums of v[0..nv) into partials[blockIdx.x * STRIDE + k] (blocks of
// at most 256 threads)
template <int NV, int STRIDE = NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], int nv, double* partials) {
  __shared__ double sh[NV][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    if (k < nv) {
      double x = v[k];
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) sh[k][w] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double s = 0.0;
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) s += sh[threadIdx.x][ww];
    partials[(size_t)blockIdx.x * STRIDE + threadIdx.x] = s;
  }
}

// The last block of a grid to finish (an arrival counter) sums the per-block
// partials of all blocks, in block order, into out[k] for k < nv and resets
// the counter: the solver kernels hand their final sums to the host without
// a separate reduction launch.  A fixed order: reproducible.
__device__ __forceinline__ void last_block_reduce(const double* partials, int stride, int nv,
                                                  unsigned* counter, double* out) {
  __shared__ unsigned s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1 ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = w; k < nv; k += nw) {
    double v = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) v += __ldcg(partials + (size_t)b * stride + k);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[k] = v;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// Element tiles of the solver kernels: a block takes 4 x 256 consecutive
// elements per step, thread t the elements t, t+256, t+512, t+768, so that
// each thread has four independent loads of every vector in flight.
constexpr int kSolU = 4, kSolT = 256;
__device__ __forceinline__ int lm_first(long long q, int nylm) { return (int)(q % nylm); }
__device__ __forceinline__ int lm_add(int lm, int d, int nylm) {
  lm += d;
  return lm >= nylm ? lm - nylm : lm;
}

// Jacobi step + DIIS Gram row: xnew = D^-1 (rhs - Ox) (jacobi_diis.f90:105-110),
// e = xnew - x (:117), dots e.h_k for the history and e.e (makeb :232-270).
// A block takes tiles of 8 x 256 consecutive elements: each thread forms
// eight elements of xnew and e and leaves e in shared memory; then warp w
// takes the history vectors k = w, w + 8, ... and reads the tile of h_k
// (sixteen loads per lane in flight) against e from shared memory.  Per
// history vector a lane accumulates in FP64 over the tiles in order, and the
// warp's shuffle tree gives the block's partial, so the row is reproducible.
// The partial row keeps the stride kMaxHist + 1 that the host-side
// reduction expects.
template <class H>
__global__ void __launch_bounds__(kSolT, 4) k_jacobi_step(const YlmTables tb, long long n,
                                                       const double* __restrict__ rhs,
                                                       const double* __restrict__ y,
                                                       const double* __restrict__ x, H* xnew,
                                                       H* e, const HistPtrs hist,
                                                       double* partials, unsigned* counter, double* out) {
  constexpr int U = 2 * kSolU;  // eight elements per thread and tile
  constexpr int TILE = U * kSolT;
  constexpr int NW = kSolT / 32;
  constexpr int KS = (kMaxHist + NW - 1) / NW;  // history vectors per warp
  constexpr int HL = 16;                        // loads per lane in flight
  __shared__ H es[TILE];
  __shared__ double red[kMaxHist + 1 + NW];
  double d[KS];
#pragma unroll
  for (int s = 0; s < KS; ++s) d[s] = 0.0;
  double ee = 0.0;
  const int nh = hist.n, nylm = tb.nylm;
  const int dt = kSolT % nylm;
  const int nn = (int)n;  // vectors hold fewer than 2^31 elements (checked at launch)
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int b0 = blockIdx.x * TILE; b0 < nn; b0 += gridDim.x * TILE) {
    const int q0 = b0 + threadIdx.x;
    int lm = lm_first(q0, nylm);
#pragma unroll
    for (int h = 0; h < U; h += kSolU) {  // two halves of four elements
      double rv[kSolU], yv[kSolU], xv[kSolU];
#pragma unroll
      for (int u = 0; u < kSolU; ++u) {
        const int q = q0 + (h + u) * kSolT;
        rv[u] = q < nn ? rhs[q] : 0.0;
        yv[u] = q < nn ? y[q] : 0.0;
        xv[u] = q < nn ? x[q] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kSolU; ++u) {
        const int q = q0 + (h + u) * kSolT;
        const double xn = tb.facl[l_of(lm)] * (rv[u] - yv[u]);
        const H ev = q < nn ? (H)(xn - xv[u]) : H(0);
        if (q < nn) {
          xnew[q] = (H)xn;
          e[q] = ev;
        }
        es[threadIdx.x + (h + u) * kSolT] = ev;
        ee = fma((double)ev, (double)ev, ee);
        lm = lm_add(lm, dt, nylm);
      }
    }
    __syncthreads();
    const int cnt = min(TILE, nn - b0);
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const int k = w + NW * s;
      if (k < nh) {
        const H* hk = static_cast<const H*>(hist.p[k]) + b0;
        for (int j0 = 0; j0 < TILE; j0 += 32 * HL) {
          H hv[HL];
#pragma unroll
          for (int u = 0; u < HL; ++u) {
            const int j = j0 + u * 32 + lane;
            hv[u] = j < cnt ? hk[j] : H(0);
          }
#pragma unroll
          for (int u = 0; u < HL; ++u)
            d[s] = fma((double)es[j0 + u * 32 + lane], (double)hv[u], d[s]);
        }
      }
    }
    __syncthreads();
  }
  // partial row [e.h_0 .. e.h_{nh-1}, e.e]
#pragma unroll
  for (int s = 0; s < KS; ++s) {
    double v = d[s];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int k = w + NW * s;
    if (lane == 0 && k < nh) red[k] = v;
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) ee += __shfl_xor_sync(0xffffffffu, ee, o);
  if (lane == 0) red[kMaxHist + 1 + w] = ee;
  __syncthreads();
  if (threadIdx.x < nh) {
    partials[(size_t)blockIdx.x * (kMaxHist + 1) + threadIdx.x] = red[threadIdx.x];
  } else if (threadIdx.x == nh) {
    double t = 0.0;
    for (int ww = 0; ww < NW; ++ww) t += red[kMaxHist + 1 + ww];
    partials[(size_t)blockIdx.x * (kMaxHist + 1) + nh] = t;
  }
  last_block_reduce(partials, kMaxHist + 1, nh + 1, counter, out);
}
// One wave: as many blocks as fit on the device at once (at most nblk, the
// partial-row capacity).
template <class KFN>
static int one_wave_blocks(KFN kfn, int nblk) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 0;
  }
  int per = 0;
  if (sms <= 0 ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, kSolT, 0) != cudaSuccess ||
      per <= 0) {
    cudaGetLastError();
    return nblk;
  }
  return std::min(nblk, sms * per);
}
template <class H>
static int jacobi_launch(Launch L, const YlmTables& tb, long long n, const double* rhs,
                         const double* y, const double* x, H* xnew, H* e, const HistPtrs& hist,
                         double* partials, int nblk, unsigned* counter, double* out) {
  const int used = one_wave_blocks(k_jacobi_step<H>, nblk);
  k_jacobi_step<H><<<used, kSolT, 0, L.st>>>(tb, n, rhs, y, x, xnew, e, hist, partials, counter,
                                             out);
  return used;
}
cudaError_t launch_jacobi_step(Launch L, const YlmTables& tb, long long n, const double* rhs,
                               const double* y, const double* x, void* xnew, void* e,
                               const HistPtrs& hist, double* partials, int nblk, bool f32,
                               int* nblk_used, unsigned* counter, double* out) {
  if (hist.n > kMaxHist - 1 || n >= (1LL << 31)) return cudaErrorInvalidValue;
  int used;
  if (f32)
    used = jacobi_launch<float>(L, tb, n, rhs, y, x, static_cast<float*>(xnew),
                                static_cast<float*>(e), hist, partials, nblk, counter, out);
  else
    used = jacobi_launch<double>(L, tb, n, rhs, y, x, static_cast<double*>(xnew),
                                 static_cast<double*>(e), hist, partials, nblk, counter, out);
  if (nblk_used) *nblk_used = used;
  ++*L.launches;
  return cudaGetLastError();
}

// DIIS extrapolation (jacobi_diis.f90:222-226) + increment norm (hnorm,
// matvec.f90:281-323: sum over spheres of sum_l 1/(l+1) |u_l|^2) + update.
template <class H>
__global__ void __launch_bounds__(kSolT) k_diis_combine(const YlmTables tb, long long n,
                                                        const HistPtrs hist,
                                                        const H* __restrict__ xjac, double* x,
                                                        double* partials, unsigned* counter, double* out) {
  double acc = 0.0;
  const int nh = hist.n, nylm = tb.nylm;
  const int dt = kSolT % nylm;
  const long long tile = (long long)kSolU * kSolT;
  for (long long b0 = (long long)blockIdx.x * tile; b0 < n; b0 += (long long)gridDim.x * tile) {
    long long q[kSolU];
    bool ok[kSolU];
    double xo[kSolU], xold[kSolU];
#pragma unroll
    for (int u = 0; u < kSolU; ++u) {
      q[u] = b0 + u * kSolT + threadIdx.x;
      ok[u] = q[u] < n;
      xold[u] = ok[u] ? x[q[u]] : 0.0;
      xo[u] = 0.0;
    }
    if (nh == 0) {
#pragma unroll
      for (int u = 0; u < kSolU; ++u) xo[u] = ok[u] ? (double)xjac[q[u]] : 0.0;
    } else {
#pragma unroll 4
      for (int k = 0; k < nh; ++k) {
        const H* hk = static_cast<const H*>(hist.p[k]);
        const double ck = hist.c[k];
        H hv[kSolU];
#pragma unroll
        for (int u = 0; u < kSolU; ++u) hv[u] = ok[u] ? hk[q[u]] : H(0);
#pragma unroll
        for (int u = 0; u < kSolU; ++u) xo[u] = fma(ck, (double)hv[u], xo[u]);
      }
    }
    int lm = lm_first(b0 + threadIdx.x, nylm);
#pragma unroll
    for (int u = 0; u < kSolU; ++u) {
      if (ok[u]) {
        const double dd = xo[u] - xold[u];
        acc = fma(dd * dd, 1.0 / (1.0 + l_of(lm)), acc);
        x[q[u]] = xo[u];
      }
      lm = lm_add(lm, dt, nylm);
    }
  }
  double v[1] = {acc};
  block_sum_store<1>(v, 1, partials);
  last_block_reduce(partials, 1, 1, counter, out);
}
cudaError_t launch_diis_combine(Launch L, const YlmTables& tb, long long n, const HistPtrs& hist,
                                const void* xjac, double* x, double* partials, int nblk,
                                bool f32, unsigned* counter, double* out) {
  if (f32)
    k_diis_combine<float><<<nblk, kSolT, 0, L.st>>>(tb, n, hist, static_cast<const float*>(xjac),
                                                    x, partials, counter, out);
  else
    k_diis_combine<double><<<nblk, kSolT, 0, L.st>>>(tb, n, hist,
                                                     static_cast<const double*>(xjac), x,
                                                     partials, counter, out);
  ++*L.launches;
  return cudaGetLastError();
}

__global__ void __launch_bounds__(256) k_hnorm_partial(const YlmTables tb, long long n,
                                                       const double* __restrict__ x,
                                                       double* partials) {
  double acc = 0.0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    int l = l_of((int)(q % tb.nylm));
    acc = fma(x[q] * x[q], 1.0 / (1.0 + l), acc);
  }
  double v[1] = {acc};
  block_sum_store<1>(v, 1, partials);
}
cudaError_t launch_hnorm_partial(Launch L, const YlmTables& tb, long long n, const double* x,
                                 double* partials, int nblk) {
  k_hnorm_partial<<<nblk, 256, 0, L.st>>>(tb, n, x, partials);
  ++*L.launches;
  return cudaGetLastError();
}

__global__ void __launch_bounds__(256) k_dot_partial(long long n, const double* __restrict__ a,
                                                     const double* __restrict__ b,
                                                     double* partials) {
  double acc = 0.0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    acc = fma(a[q], b[q], acc);
  double v[1] = {acc};
  block_sum_store<1>(v, 1, partials);
}
cudaError_t launch_dot_partial(Launch L, long long n, const double* a, const double* b,
                               double* partials, int nblk) {
  k_dot_partial<<<nblk, 256, 0, L.st>>>(n, a, b, partials);
  ++*L.launches;
  return cudaGetLastError();
}

// out[k] = sum over blocks of partials[b][k] in a fixed tree order
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblk, int stride,
                                  double* out) {
  __shared__ double sh[256];
  const int k = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += 256) s += partials[(size_t)b * stride + k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h >= 1; h >>= 1) {
    if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = sh[0];
}
cudaError_t launch_reduce_partials(Launch L, const double* partials, int nblk, int nvals,
                                   int stride, double* out) {
  if (nvals > stride) return cudaErrorInvalidValue;
  k_reduce_partials<<<nvals, 256, 0, L.st>>>(partials, nblk, stride, out);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// solute electrostatics (mkrhs.f90:100-120, efld.f90:97-114): direct sums
// with source tiles staged in shared memory, summed in source order.
// ---------------------------------------------------------------------------
constexpr int kNbTile = 256;
// Source range of each thread's target ([0, nsrc) for one molecule; the
// target's own molecule in a batch) and the union over the block.
struct SrcRange {
  int lo, hi, ulo, uhi;
};
__device__ __forceinline__ SrcRange block_src_range(const int2* trange, int t, int ntrg,
                                                    int s0, int s1) {
  __shared__ int b_lo, b_hi;
  SrcRange r;
  r.lo = s0;
  r.hi = s1;
  if (trange) {
    if (t < ntrg) {
      int2 v = trange[t];
      r.lo = max(v.x, s0);
      r.hi = min(v.y, s1);
    } else {
      r.lo = s1;
      r.hi = s0;
    }
  }
  if (threadIdx.x == 0) {
    b_lo = s1;
    b_hi = s0;
  }
  __syncthreads();
  if (r.lo < r.hi) {
    atomicMin(&b_lo, r.lo);
    atomicMax(&b_hi, r.hi);
  }
  __syncthreads();
  r.ulo = b_lo;
  r.uhi = b_hi;
  return r;
}

__global__ void __launch_bounds__(kNbTile) k_coulomb_pot(int nsrc, const double* __restrict__ q,
                                                         const double* __restrict__ sx,
                                                         const double* __restrict__ sy,
                                                         const double* __restrict__ sz,
                                                         int ntrg, const double* __restrict__ ctrg,
                                                         double* phi,
                                                         const int2* __restrict__ trange) {
  __shared__ double4 src[kNbTile];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double px = 0, py = 0, pz = 0;
  if (t < ntrg) {
    px = ctrg[3 * (size_t)t];
    py = ctrg[3 * (size_t)t + 1];
    pz = ctrg[3 * (size_t)t + 2];
  }
  const SrcRange rg = block_src_range(trange, t, ntrg, 0, nsrc);
  double v = 0.0;
  for (int j0 = rg.ulo; j0 < rg.uhi; j0 += kNbTile) {
    int j = j0 + threadIdx.x;
    __syncthreads();
    src[threadIdx.x] = j < rg.uhi ? make_double4(sx[j], sy[j], sz[j], q[j])
                                  : make_double4(0, 0, 0, 0);
    __syncthreads();
    int cnt = min(kNbTile, rg.uhi - j0);
    const int kb = max(rg.lo - j0, 0), ke = min(rg.hi - j0, cnt);
    if (kb == 0 && ke == kNbTile) {
#pragma unroll 8
      for (int k = 0; k < kNbTile; ++k) {
        double4 s = src[k];
        double dx = px - s.x, dy = py - s.y, dz = pz - s.z;
        v = fma(s.w, rsqrt_pos(dx * dx + dy * dy + dz * dz), v);
      }
    } else {
      for (int k = kb; k < ke; ++k) {
        double4 s = src[k];
        double dx = px - s.x, dy = py - s.y, dz = pz - s.z;
        v = fma(s.w, rsqrt_pos(dx * dx + dy * dy + dz * dz), v);
      }
    }
  }
  if (t < ntrg) phi[t] = v;
}
// The potential and, for the forces, the solute's field at the same targets
// (efld.f90:97-114 with the nuclei as sources) from one pass over the pairs:
// per pair the field adds q r^-3 (p - s) to the potential's q r^-1.
__global__ void __launch_bounds__(kNbTile) k_coulomb_pot_field(
    int nsrc, const double* __restrict__ q, const double* __restrict__ sx,
    const double* __restrict__ sy, const double* __restrict__ sz, int ntrg,
    const double* __restrict__ ctrg, double* phi, double* ef, const int2* __restrict__ trange) {
  __shared__ double4 src[kNbTile];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double px = 0, py = 0, pz = 0;
  if (t < ntrg) {
    px = ctrg[3 * (size_t)t];
    py = ctrg[3 * (size_t)t + 1];
    pz = ctrg[3 * (size_t)t + 2];
  }
  const SrcRange rg = block_src_range(trange, t, ntrg, 0, nsrc);
  double v = 0.0, ex = 0.0, ey = 0.0, ez = 0.0;
  auto pair = [&](const double4& s) {
    const double dx = px - s.x, dy = py - s.y, dz = pz - s.z;
    const double ri = rsqrt_pos(dx * dx + dy * dy + dz * dz);
    v = fma(s.w, ri, v);
    const double f = s.w * (ri * ri * ri);
    ex = fma(f, dx, ex);
    ey = fma(f, dy, ey);
    ez = fma(f, dz, ez);
  };
  for (int j0 = rg.ulo; j0 < rg.uhi; j0 += kNbTile) {
    int j = j0 + threadIdx.x;
    __syncthreads();
    src[threadIdx.x] = j < rg.uhi ? make_double4(sx[j], sy[j], sz[j], q[j])
                                  : make_double4(0, 0, 0, 0);
    __syncthreads();
    int cnt = min(kNbTile, rg.uhi - j0);
    const int kb = max(rg.lo - j0, 0), ke = min(rg.hi - j0, cnt);
    if (kb == 0 && ke == kNbTile) {
#pragma unroll 4
      for (int k = 0; k < kNbTile; ++k) pair(src[k]);
    } else {
      for (int k = kb; k < ke; ++k) pair(src[k]);
    }
  }
  if (t < ntrg) {
    phi[t] = v;
    ef[3 * (size_t)t] = ex;
    ef[3 * (size_t)t + 1] = ey;
    ef[3 * (size_t)t + 2] = ez;
  }
}
cudaError_t launch_coulomb_pot_field(Launch L, int nsrc, const double* q, const double* sx,
                                     const double* sy, const double* sz, int ntrg,
                                     const double* ctrg, double* phi, double* ef,
                                     const int2* trange) {
  if (ntrg == 0) return cudaSuccess;
  k_coulomb_pot_field<<<(ntrg + kNbTile - 1) / kNbTile, kNbTile, 0, L.st>>>(
      nsrc, q, sx, sy, sz, ntrg, ctrg, phi, ef, trange);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_coulomb_pot(Launch L, int nsrc, const double* q, const double* sx,
                               const double* sy, const double* sz, int ntrg, const double* ctrg,
                               double* phi, const int2* trange) {
  if (ntrg == 0) return cudaSuccess;
  k_coulomb_pot<<<(ntrg + kNbTile - 1) / kNbTile, kNbTile, 0, L.st>>>(nsrc, q, sx, sy, sz, ntrg,
                                                                       ctrg, phi, trange);
  ++*L.launches;
  return cudaGetLastError();
}
__global__ void k_psi(int n, int nylm, const double* __restrict__ q, double* psi) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * nylm) return;
  int i = (int)(e / nylm), lm = (int)(e - (long long)i * nylm);
  psi[e] = lm == 0 ? sqrt(16.0 * atan(1.0)) * q[i] : 0.0;
}
cudaError_t launch_psi(Launch L, int n, int nylm, const double* q, double* psi) {
  long long np = (long long)n * nylm;
  if (np == 0) return cudaSuccess;
  k_psi<<<(unsigned)((np + 255) / 256), 256, 0, L.st>>>(n, nylm, q, psi);
  ++*L.launches;
  return cudaGetLastError();
}

int efield_chunks(int nsrc, int ntrg) {
  int tiles = (ntrg + kNbTile - 1) / kNbTile;
  int want = (148 * 8 + tiles - 1) / max(tiles, 1);
  int maxc = (nsrc + 4 * kNbTile - 1) / (4 * kNbTile);
  return max(1, min(want, max(maxc, 1)));
}
// source chunks for the FP32 field of one molecule: enough blocks of the
// two-targets-per-thread kernel (k_efield_f2) to fill the device
int efield_chunks_f32(int nsrc, int ntrg) {
  int tiles2 = (ntrg + 2 * kNbTile - 1) / (2 * kNbTile);
  int want = (148 * 8 + tiles2 - 1) / max(tiles2, 1);
  int maxc = (nsrc + 4 * kNbTile - 1) / (4 * kNbTile);
  return max(1, min(want, max(maxc, 1)));
}

__global__ void __launch_bounds__(kNbTile) k_efield(int nsrc, const double* __restrict__ q,
                                                    const double* __restrict__ csrc, int ntrg,
                                                    const double* __restrict__ ctrg, int chunk,
                                                    double* out,
                                                    const int2* __restrict__ trange) {
  __shared__ double4 src[kNbTile];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  double px = 0, py = 0, pz = 0;
  if (t < ntrg) {
    px = ctrg[3 * (size_t)t];
    py = ctrg[3 * (size_t)t + 1];
    pz = ctrg[3 * (size_t)t + 2];
  }
  double ex = 0.0, ey = 0.0, ez = 0.0;
  const SrcRange rg = block_src_range(trange, t, ntrg, c * chunk, min(nsrc, c * chunk + chunk));
  for (int j0 = rg.ulo; j0 < rg.uhi; j0 += kNbTile) {
    int j = j0 + threadIdx.x;
    __syncthreads();
    src[threadIdx.x] = j < rg.uhi ? make_double4(csrc[3 * (size_t)j], csrc[3 * (size_t)j + 1],
                                                 csrc[3 * (size_t)j + 2], q[j])
                                  : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int cnt = min(kNbTile, rg.uhi - j0);
    const int kb = max(rg.lo - j0, 0), ke = min(rg.hi - j0, cnt);
#pragma unroll 4
    for (int k = kb; k < ke; ++k) {
      double4 s = src[k];
      double dx = px - s.x, dy = py - s.y, dz = pz - s.z;
      double r2 = dx * dx + dy * dy + dz * dz;
      double ri = rsqrt_pos(r2);
      double f = s.w * (ri * ri * ri);
      ex = fma(f, dx, ex);
      ey = fma(f, dy, ey);
      ez = fma(f, dz, ez);
    }
  }
  if (t < ntrg) {
    double* o = out + ((size_t)c * ntrg + t) * 3;
    o[0] = ex;
    o[1] = ey;
    o[2] = ez;
  }
}
__global__ void k_efield_reduce(int ntrg, int nchunk, const double* __restrict__ scratch,
                                double* ef) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3LL * ntrg) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; ++c) s += scratch[(size_t)c * 3 * ntrg + e];
  ef[e] = s;
}
// FP32-pair variant (mixed precision, force terms only): coordinates are
// taken relative to the block's first target in FP64 and rounded once to
// FP32; each 256-source tile is summed in FP32 and added to FP64
// accumulators.  Same chunked partial-sum layout as k_efield.
__global__ void __launch_bounds__(kNbTile) k_efield_f(int nsrc, const double* __restrict__ q,
                                                      const double* __restrict__ csrc, int ntrg,
                                                      const double* __restrict__ ctrg, int chunk,
                                                      double* out,
                                                      const int2* __restrict__ trange) {
  __shared__ float4 src[kNbTile];
  __shared__ double org[3];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (threadIdx.x == 0) {
    int t0 = blockIdx.x * blockDim.x;
    org[0] = ctrg[3 * (size_t)t0];
    org[1] = ctrg[3 * (size_t)t0 + 1];
    org[2] = ctrg[3 * (size_t)t0 + 2];
  }
  __syncthreads();
  const double ox = org[0], oy = org[1], oz = org[2];
  float px = 0.f, py = 0.f, pz = 0.f;
  if (t < ntrg) {
    px = (float)(ctrg[3 * (size_t)t] - ox);
    py = (float)(ctrg[3 * (size_t)t + 1] - oy);
    pz = (float)(ctrg[3 * (size_t)t + 2] - oz);
  }
  double ex = 0.0, ey = 0.0, ez = 0.0;
  const SrcRange rg = block_src_range(trange, t, ntrg, c * chunk, min(nsrc, c * chunk + chunk));
  for (int j0 = rg.ulo; j0 < rg.uhi; j0 += kNbTile) {
    int j = j0 + threadIdx.x;
    __syncthreads();
    src[threadIdx.x] = j < rg.uhi ? make_float4((float)(csrc[3 * (size_t)j] - ox),
                                                (float)(csrc[3 * (size_t)j + 1] - oy),
                                                (float)(csrc[3 * (size_t)j + 2] - oz),
                                                (float)q[j])
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    const int cnt = min(kNbTile, rg.uhi - j0);
    const int kb = max(rg.lo - j0, 0), ke = min(rg.hi - j0, cnt);
    float fx = 0.f, fy = 0.f, fz = 0.f;
#pragma unroll 8
    for (int k = kb; k < ke; ++k) {
      float4 s = src[k];
      float dx = px - s.x, dy = py - s.y, dz = pz - s.z;
      float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      float ri = rsqrtf(r2);
      float f = s.w * (ri * ri * ri);
      fx = fmaf(f, dx, fx);
      fy = fmaf(f, dy, fy);
      fz = fmaf(f, dz, fz);
    }
    ex += fx;
    ey += fy;
    ez += fz;
  }
  if (t < ntrg) {
    double* o = out + ((size_t)c * ntrg + t) * 3;
    o[0] = ex;
    o[1] = ey;
    o[2] = ez;
  }
}
// One molecule: two targets per thread (targets t and t + kNbTile of a
// 2*kNbTile block), so each broadcast source read serves both.  Same
// arithmetic per pair and the same summation order per target as k_efield_f.
__global__ void __launch_bounds__(kNbTile) k_efield_f2(int nsrc, const double* __restrict__ q,
                                                       const double* __restrict__ csrc, int ntrg,
                                                       const double* __restrict__ ctrg,
                                                       int chunk, double* out) {
  __shared__ float4 src[kNbTile];
  const int tb0 = blockIdx.x * 2 * kNbTile;
  const int c = blockIdx.y;
  const double ox = ctrg[3 * (size_t)tb0], oy = ctrg[3 * (size_t)tb0 + 1],
               oz = ctrg[3 * (size_t)tb0 + 2];
  float p[2][3];
  int tt[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int t = tb0 + h * kNbTile + threadIdx.x;
    tt[h] = t;
    p[h][0] = p[h][1] = p[h][2] = 0.f;
    if (t < ntrg) {
      p[h][0] = (float)(ctrg[3 * (size_t)t] - ox);
      p[h][1] = (float)(ctrg[3 * (size_t)t + 1] - oy);
      p[h][2] = (float)(ctrg[3 * (size_t)t + 2] - oz);
    }
  }
  double e[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  const int s0 = c * chunk, s1 = min(nsrc, c * chunk + chunk);
  for (int j0 = s0; j0 < s1; j0 += kNbTile) {
    const int j = j0 + threadIdx.x;
    __syncthreads();
    src[threadIdx.x] = j < s1 ? make_float4((float)(csrc[3 * (size_t)j] - ox),
                                            (float)(csrc[3 * (size_t)j + 1] - oy),
                                            (float)(csrc[3 * (size_t)j + 2] - oz), (float)q[j])
                              : make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    const int cnt = min(kNbTile, s1 - j0);
    float f[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll 4
    for (int k = 0; k < cnt; ++k) {
      const float4 sv = src[k];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float dx = p[h][0] - sv.x, dy = p[h][1] - sv.y, dz = p[h][2] - sv.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float ri = rsqrtf(r2);
        const float w = sv.w * (ri * ri * ri);
        f[h][0] = fmaf(w, dx, f[h][0]);
        f[h][1] = fmaf(w, dy, f[h][1]);
        f[h][2] = fmaf(w, dz, f[h][2]);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      e[h][0] += f[h][0];
      e[h][1] += f[h][1];
      e[h][2] += f[h][2];
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h)
    if (tt[h] < ntrg) {
      double* o = out + ((size_t)c * ntrg + tt[h]) * 3;
      o[0] = e[h][0];
      o[1] = e[h][1];
      o[2] = e[h][2];
    }
}

cudaError_t launch_efield_f32(Launch L, int nsrc, const double* q, const double* csrc, int ntrg,
                              const double* ctrg, double* ef, double* scratch, int nchunk,
                              const int2* trange) {
  if (ntrg == 0) return cudaSuccess;
  int chunk = (nsrc + nchunk - 1) / max(nchunk, 1);
  chunk = ((chunk + kNbTile - 1) / kNbTile) * kNbTile;
  if (chunk == 0) chunk = kNbTile;
  double* out = nchunk == 1 ? ef : scratch;
  const int tiles2 = (ntrg + 2 * kNbTile - 1) / (2 * kNbTile);
  if (!trange && (long long)tiles2 * nchunk >= 148 * 8) {  // enough blocks to fill the GPU
    dim3 grid2(tiles2, nchunk);
    k_efield_f2<<<grid2, kNbTile, 0, L.st>>>(nsrc, q, csrc, ntrg, ctrg, chunk, out);
  } else {
    dim3 grid((ntrg + kNbTile - 1) / kNbTile, nchunk);
    k_efield_f<<<grid, kNbTile, 0, L.st>>>(nsrc, q, csrc, ntrg, ctrg, chunk, out, trange);
  }
  ++*L.launches;
  cudaError_t e = cudaGetLastError();
  if (e || nchunk == 1) return e;
  k_efield_reduce<<<(unsigned)((3LL * ntrg + 255) / 256), 256, 0, L.st>>>(ntrg, nchunk, scratch, ef);
  ++*L.launches;
  return cudaGetLastError();
}

cudaError_t launch_efield(Launch L, int nsrc, const double* q, const double* csrc, int ntrg,
                          const double* ctrg, double* ef, double* scratch, int nchunk,
                          const int2* trange) {
  if (ntrg == 0) return cudaSuccess;
  int chunk = (nsrc + nchunk - 1) / max(nchunk, 1);
  chunk = ((chunk + kNbTile - 1) / kNbTile) * kNbTile;
  if (chunk == 0) chunk = kNbTile;
  dim3 grid((ntrg + kNbTile - 1) / kNbTile, nchunk);
  double* out = nchunk == 1 ? ef : scratch;
  k_efield<<<grid, kNbTile, 0, L.st>>>(nsrc, q, csrc, ntrg, ctrg, chunk, out, trange);
  ++*L.launches;
  cudaError_t e = cudaGetLastError();
  if (e || nchunk == 1) return e;
  k_efield_reduce<<<(unsigned)((3LL * ntrg + 255) / 256), 256, 0, L.st>>>(ntrg, nchunk, scratch, ef);
  ++*L.launches;
  return cudaGetLastError();
}
// Loads the FP64 field kernels' code onto the current device now, rather than
// at their first launch (CUDA loads modules lazily by default).
cudaError_t preload_efield() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k_efield);
  if (e != cudaSuccess) return e;
  return cudaFuncGetAttributes(&a, k_efield_reduce);
}

// ---------------------------------------------------------------------------
// forces (fdoka ddcosmo.f90:1436-1504, fdokb :1511-1607, fdoga :1614-1650)
// ---------------------------------------------------------------------------
// alp = sum_{l>=1} t^{l-1}/facl_l sum_m sig_lm (l Y_lm s + dY_lm) and
// beta = sum_l t^l/facl_l sum_m sig_lm Y_lm, with Y and its surface gradient
// as dbasis (ddcosmo.f90:904-1043) computes them, pole branches included.
template <int LMAX>
__device__ void dbasis_contract(const YlmTables& tb, double sx, double sy, double sz, double t,
                                const double* __restrict__ sig, double alp[3], double& beta) {
  constexpr int NY = (LMAX + 1) * (LMAX + 1);
  double vplm[NY];
  double vc[LMAX + 2], vs[LMAX + 2];
  double cthe = sz;
  double sthe = sqrt(fmax(0.0, 1.0 - cthe * cthe));
  double cphi, sphi, et[3], ep[3];
  const bool pole = !(sthe != 0.0);
  if (!pole) {
    cphi = sx / sthe;
    sphi = sy / sthe;
  } else {
    cphi = 1.0;
    sphi = 0.0;
  }
  et[0] = cthe * cphi;
  et[1] = cthe * sphi;
  et[2] = -sthe;
  if (!pole) {
    ep[0] = -sphi / sthe;
    ep[1] = cphi / sthe;
  } else {
    ep[0] = 0.0;
    ep[1] = 1.0;
  }
  ep[2] = 0.0;
  vc[0] = 1.0; vs[0] = 0.0;
  if (!pole) {
    vc[1] = cphi; vs[1] = sphi;
    for (int m = 2; m <= LMAX; ++m) {
      vc[m] = 2.0 * cphi * vc[m - 1] - vc[m - 2];
      vs[m] = 2.0 * cphi * vs[m - 1] - vs[m - 2];
    }
  } else {
    for (int m = 1; m <= LMAX; ++m) { vc[m] = 1.0; vs[m] = 0.0; }
  }
  const double VC = 0.0, VS = (double)(int)cthe;  // integer VC/VS (ddcosmo.f90:912)
  {  // polleg
    double fact = 1.0, pmm = 1.0;
    for (int m = 0; m <= LMAX; ++m) {
      int ind = (m + 1) * (m + 1) - 1;
      vplm[ind] = pmm;
      if (m == LMAX) break;
      double pmm1 = cthe * (2.0 * m + 1.0) * pmm;
      vplm[ind + 2 * m + 2] = pmm1;
      double pmmo = pmm;
      for (int l = m + 2; l <= LMAX; ++l) {
        double pll = tb.A[lmi(l, m)] * cthe * pmm1 - tb.B[lmi(l, m)] * pmm;
        vplm[l * l + l + m] = pll;
        pmm = pmm1;
        pmm1 = pll;
      }
      pmm = -pmmo * fact * sthe;
      fact += 2.0;
    }
  }
  alp[0] = alp[1] = alp[2] = 0.0;
  beta = 0.0;
  double tl = 1.0;  // t^l
  for (int l = 0; l <= LMAX; ++l) {
    const int ind = l * l + l;
    const double fl = (double)l;
    double bl = 0.0, a0 = 0.0, a1 = 0.0, a2 = 0.0;
    {
      double fln = tb.facs[lmi(l, 0)];
      double Y = fln * vplm[ind];
      double sg = sig[ind];
      bl += Y * sg;
      if (l > 0) {
        double d = fln * vplm[ind + 1];
        a0 += sg * (fl * Y * sx + d * et[0]);
        a1 += sg * (fl * Y * sy + d * et[1]);
        a2 += sg * (fl * Y * sz + d * et[2]);
      }
    }
    for (int m = 1; m <= l; ++m) {
      double fln = tb.facs[lmi(l, m)];
      double plm = fln * vplm[ind + m];
      double pp1 = (m < l) ? -0.5 * vplm[ind + m + 1] : 0.0;
      double pm1 = 0.5 * ((double)(l + m) * (double)(l - m + 1) * vplm[ind + m - 1]);
      double pp = pp1 + pm1;
      double Yc = plm * vc[m], Ys = plm * vs[m];
      double dc[3], ds[3];
      for (int k = 0; k < 3; ++k) {
        if (!pole) {
          dc[k] = -fln * pp * vc[m] * et[k] - (double)m * plm * vs[m] * ep[k];
          ds[k] = -fln * pp * vs[m] * et[k] + (double)m * plm * vc[m] * ep[k];
        } else {
          dc[k] = -fln * pp * vc[m] * et[k] - fln * pp * ep[k] * VC;
          ds[k] = -fln * pp * vs[m] * et[k] - fln * pp * ep[k] * VS;
        }
      }
      double sc = sig[ind + m], ss = sig[ind - m];
      bl += Yc * sc + Ys * ss;
      a0 += sc * (fl * Yc * sx + dc[0]) + ss * (fl * Ys * sx + ds[0]);
      a1 += sc * (fl * Yc * sy + dc[1]) + ss * (fl * Ys * sy + ds[1]);
      a2 += sc * (fl * Yc * sz + dc[2]) + ss * (fl * Ys * sz + ds[2]);
    }
    const double ifl = 1.0 / tb.facl[l];
    if (l >= 1) {
      double f = (tl / t) * ifl;  // t^{l-1}/facl_l
      if (t == 0.0) f = (l == 1) ? ifl : 0.0;
      alp[0] += f * a0;
      alp[1] += f * a1;
      alp[2] += f * a2;
    }
    beta += tl * ifl * bl;
    tl *= t;
  }
}

// The same alp and beta from the recurrence of the fused L / L* pass.  With
// u = v / r_i (|u| = t, u / |u| = s) and the real solid harmonics
// R_lm(u) = t^l Y_lm(s), the contraction above is
//   beta  = sum_lm w_lm R_lm(u),   alp_k = sum_lm w_lm d_k R_lm(u),
// w = sigma / facl, and d_k R_lm is a harmonic polynomial of degree l - 1,
// so alp_k = sum_{l'm'} G^k_{l'm'} R_{l'm'}(u) with l' = l - 1.  G follows
// from the ladder relations of the complex solid harmonics without the
// Condon-Shortley phase, S_l^m = |u|^l Pt_l^m(cos theta) e^{i m phi}:
//   d_z S_l^m = (l+m) S_{l-1}^m,   (d_x + i d_y) S_l^m = -S_{l-1}^{m+1},
//   (d_x - i d_y) S_l^m = (l+m)(l+m-1) S_{l-1}^{m-1}   (m >= 1),
//   (d_x - i d_y) S_l^0 = -conj(S_{l-1}^1),
// with R_{l,+m} = nu_lm Re S_l^m, R_{l,-m} = nu_lm Im S_l^m, nu_lm = |facs_lm|.
// k_force_vec writes per sphere the four vectors (beta, G^x, G^y, G^z) in
// the (l, m >= 0) pair layout, scaled by Kg facl so that they contract the
// normalised recurrence values Q_l^m (prefix 1) times cos / sin m phi.
template <int LMAX>
__global__ void k_force_vec(const YlmTables tb, int nsph, const double* __restrict__ sigma,
                            double2* __restrict__ fv) {
  constexpr int NLM = (LMAX + 1) * (LMAX + 2) / 2;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)nsph * NLM) return;
  const int i = (int)(e / NLM), le = (int)(e - (long long)i * NLM);
  int lp = 0;
  while (lmi(lp + 1, 0) <= le) ++lp;
  const int m = le - lmi(lp, 0);
  const double* sg = sigma + (size_t)i * tb.nylm;
  auto nu = [&](int l, int mm) { return fabs(tb.facs[lmi(l, mm)]); };
  auto wc = [&](int l, int mm) { return sg[l * l + l + mm] / tb.facl[l]; };
  auto ws = [&](int l, int mm) { return sg[l * l + l - mm] / tb.facl[l]; };
  double2* out = fv + 4 * (size_t)e;
  out[0] = make_double2(tb.Kg[le] * sg[lp * lp + lp + m], m ? tb.Kg[le] * sg[lp * lp + lp - m] : 0.0);
  double gxc = 0.0, gxs = 0.0, gyc = 0.0, gys = 0.0, gzc = 0.0, gzs = 0.0;
  if (lp < LMAX) {
    const int l = lp + 1;
    gzc = (double)(l + m) * nu(l, m) * wc(l, m);
    if (m >= 1) gzs = (double)(l + m) * nu(l, m) * ws(l, m);
    if (m + 1 <= l) {  // lowering from m + 1
      const double f = 0.5 * nu(l, m + 1) * ((double)(l + m + 1) * (double)(l + m));
      gxc += f * wc(l, m + 1);
      gyc += f * ws(l, m + 1);
      if (m >= 1) {
        gxs += f * ws(l, m + 1);
        gys -= f * wc(l, m + 1);
      }
    }
    if (m >= 2) {  // raising from m - 1
      const double f = 0.5 * nu(l, m - 1);
      gxc -= f * wc(l, m - 1);
      gyc += f * ws(l, m - 1);
      gxs -= f * ws(l, m - 1);
      gys -= f * wc(l, m - 1);
    } else if (m == 1) {  // raising from m = 0
      gxc -= nu(l, 0) * wc(l, 0);
      gys -= nu(l, 0) * wc(l, 0);
    }
    const double sc = tb.Kg[le] * tb.facl[lp] / nu(lp, m);
    gxc *= sc; gxs *= sc; gyc *= sc; gys *= sc; gzc *= sc; gzs *= sc;
  }
  out[1] = make_double2(gxc, gxs);
  out[2] = make_double2(gyc, gys);
  out[3] = make_double2(gzc, gzs);
}
cudaError_t launch_force_vec(Launch L, const YlmTables& tb, int nsph, const double* sigma,
                             double2* fv) {
  const int nlm = (tb.lmax + 1) * (tb.lmax + 2) / 2;
  const long long n = (long long)nsph * nlm;
  if (n == 0) return cudaSuccess;
#define CASE(LV)                                                                              \
  case LV:                                                                                    \
    k_force_vec<LV><<<(unsigned)((n + 127) / 128), 128, 0, L.st>>>(tb, nsph, sigma, fv);       \
    break;
  switch (tb.lmax) {
    DDC_LMAX_CASES(CASE)
    default:
      return cudaErrorInvalidValue;
  }
#undef CASE
  ++*L.launches;
  return cudaGetLastError();
}
// beta and alp of one triple (s off the poles) from the vectors V of its
// sphere: ct = t cos theta, t2 = t^2, st = t sin theta, (cp, sp) = (cos, sin)
// phi.  The column loop is not unrolled (register pressure); (l, m) is warp
// uniform, so the table and shared-memory reads are broadcasts.
template <int LMAX>
__device__ __forceinline__ void force_contract(const YlmTables& tb, double ct, double t2,
                                               double st, double cp, double sp,
                                               const double2* V, double alp[3], double& beta) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  double pmm = 1.0, cm = 1.0, sm = 0.0, cmm1 = 1.0, smm1 = 0.0;
#pragma unroll 1
  for (int m = 0; m <= LMAX; ++m) {
    if (m == 1) {
      cm = cp;
      sm = sp;
    } else if (m >= 2) {
      const double cn = 2.0 * cp * cm - cmm1, sn = 2.0 * cp * sm - smm1;
      cmm1 = cm; smm1 = sm; cm = cn; sm = sn;
    }
    double dc[4] = {0.0, 0.0, 0.0, 0.0}, ds[4] = {0.0, 0.0, 0.0, 0.0};
    // value Q of degree l: beta for every l, the gradient vectors below lmax
    auto add = [&](double Q, int l) {
      const double2* v = V + 4 * lmi(l, m);
      const int nv = l < LMAX ? 4 : 1;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (k < nv) {
          const double2 c = v[k];
          dc[k] = fma(Q, c.x, dc[k]);
          ds[k] = fma(Q, c.y, ds[k]);
        }
    };
    double q0 = pmm, q1 = ct * pmm;
    add(q0, m);
    if (m < LMAX) {
      add(q1, m + 1);
#pragma unroll 2
      for (int l = m + 2; l <= LMAX; ++l) {
        const double Q = fma(ct, q1, -(tb.Bn[lmi(l, m)] * t2) * q0);
        q0 = q1;
        q1 = Q;
        add(Q, l);
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] = fma(cm, dc[k], fma(sm, ds[k], acc[k]));
    pmm = -pmm * (double)(2 * m + 1) * st;
  }
  beta = acc[0];
  alp[0] = acc[1];
  alp[1] = acc[2];
  alp[2] = acc[3];
}

// Forces, kernel A: block per sphere i over its gather list, i.e. the
// triples (j, n, i) with point n of neighbour j inside i.  fdoka(j)
// (ddcosmo.f90:1436-1504) and fdokb(i) (:1511-1607) both contract
// dbasis(s_n^ji) with sigma_i at such a triple, so alp and beta are computed
// once per triple: the fdokb and fdoga-neighbour terms accumulate into
// fxa(:,i), the fdoka term of sphere j goes to the per-triple slot fda(:,q).
// fdokb's inner loop over k in N_j (:1575-1590) is u_chi(j,n) - chi_ji*beta
// with u_chi = sum_k chi_jk intmlp_k (an extra k_lx pass on sigma).
// alp and beta come from force_contract off the poles and from the
// reference's dbasis restatement at them.
template <int LMAX>
__global__ void __launch_bounds__(128) k_forces_a(const YlmTables tb, const DevGeo g,
                                                  const double* __restrict__ sigma,
                                                  const double2* __restrict__ fv,
                                                  const double* __restrict__ xs,
                                                  const double* __restrict__ uchi,
                                                  const double* __restrict__ phi, double* fxa,
                                                  double* fda) {
  constexpr int NLM = (LMAX + 1) * (LMAX + 2) / 2;
  __shared__ double2 sv[4 * NLM];
  const int i = blockIdx.x;
  for (int k = threadIdx.x; k < 4 * NLM; k += blockDim.x) sv[k] = fv[4 * (size_t)i * NLM + k];
  __syncthreads();
  const int G = g.ngrid, NY = g.nylm;
  const double4 ci = g.sph[i];
  const double eta = tb.eta, tlow = 1.0 - eta;
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double* si = sigma + (size_t)i * NY;
  for (int q = g.ls_ptr[i] + threadIdx.x; q < g.ls_ptr[i + 1]; q += blockDim.x) {
    const int2 jn = g.ls[q];
    const int j = jn.x, n = jn.y;
    const double4 cj = g.sph[j];
    const double4 gn = g.grid[n];
    const size_t pj = (size_t)j * G + n;
    Rel r = rel_exact(cj, gn, ci);
    double sx = r.vx / r.vv, sy = r.vy / r.vv, sz = r.vz / r.vv;
    double alp[3], beta;
    const double sthe = sqrt(fmax(0.0, 1.0 - sz * sz));
    if (sthe != 0.0)
      force_contract<LMAX>(tb, r.t * sz, r.t * r.t, r.t * sthe, sx / sthe, sy / sthe, sv, alp,
                           beta);
    else
      dbasis_contract<LMAX>(tb, sx, sy, sz, r.t, si, alp, beta);
    double xji = fsw_exact(r.t, eta), fj = g.fi[pj];
    double xij = xs[pj];
    double dsw = (r.t > tlow) ? dfsw_exact(r.t, eta) : 0.0;
    // fdoka term of sphere j at its point n (neighbour i): -w xi_j(n) va
    {
      double oij, fb;
      if (fj > 1.0) {
        oij = xji / fj;
        fb = -oij / fj;
      } else {
        oij = xji;
        fb = 0.0;
      }
      double fa = oij / ci.w;
      double va0 = fa * alp[0] + beta * fb * g.zi[3 * pj];
      double va1 = fa * alp[1] + beta * fb * g.zi[3 * pj + 1];
      double va2 = fa * alp[2] + beta * fb * g.zi[3 * pj + 2];
      if (r.t > tlow) {
        double f3 = beta * dsw / ci.w;
        if (fj > 1.0) f3 = f3 / fj;
        va0 += f3 * sx;
        va1 += f3 * sy;
        va2 += f3 * sz;
      }
      double c = -gn.w * xij;
      fda[3 * (size_t)q + 0] = c * va0;
      fda[3 * (size_t)q + 1] = c * va1;
      fda[3 * (size_t)q + 2] = c * va2;
    }
    // fdokb and the neighbour part of fdoga for sphere i
    double oji = fj > 1.0 ? xji / fj : xji;
    double fa = oji / ci.w;
    double vb0 = fa * alp[0] * xij, vb1 = fa * alp[1] * xij, vb2 = fa * alp[2] * xij;
    double vc0 = 0.0, vc1 = 0.0, vc2 = 0.0;
    if (r.t > tlow) {
      double di, fac;
      if (fj > 1.0) {
        di = 1.0 / fj;
        fac = di * xji;
        if (g.ntri_pt[pj] >= 2) {
          double b = uchi[pj] - xji * beta;
          double g1 = di * di * dsw / ci.w;
          double g2 = g1 * xij * b;
          vc0 = g2 * sx;
          vc1 = g2 * sy;
          vc2 = g2 * sz;
        }
      } else {
        di = 1.0;
        fac = 0.0;
      }
      double fb2 = (1.0 - fac) * di * dsw / ci.w;
      vb0 += fb2 * xij * beta * sx;
      vb1 += fb2 * xij * beta * sy;
      vb2 += fb2 * xij * beta * sz;
      if (r.t < 1.0 && g.ui[pj] > 0.0) {
        int cidx = g.cavidx[pj];
        double ph = cidx >= 0 ? phi[cidx] : 0.0;
        double fg = dsw / ci.w * ph * xij;
        vb0 += fg * sx;
        vb1 += fg * sy;
        vb2 += fg * sz;
      }
    }
    f0 += gn.w * (vb0 - vc0);
    f1 += gn.w * (vb1 - vc1);
    f2 += gn.w * (vb2 - vc2);
  }
  __shared__ double sh[3][4];
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    f0 += __shfl_xor_sync(0xffffffffu, f0, o);
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
  }
  if (lane == 0) {
    sh[0][w] = f0;
    sh[1][w] = f1;
    sh[2][w] = f2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int ww = 0; ww < nw; ++ww) s += sh[threadIdx.x][ww];
    fxa[3 * (size_t)i + threadIdx.x] = s;
  }
}

// Forces, kernel B: block per sphere j.  Sums the fdoka slots of j (its pair
// lists, found through lsstart), the fdoga point term (0 < U < 1) and the
// kernel-A part, in fixed order, and applies fep (forces_dd.f90:160-161).
__global__ void __launch_bounds__(128) k_forces_b(const DevGeo g, const double* __restrict__ xs,
                                                  const double* __restrict__ phi,
                                                  const double* __restrict__ fxa,
                                                  const double* __restrict__ fda,
                                                  const int* __restrict__ lsstart, double fep,
                                                  double* fx) {
  const int j = blockIdx.x;
  const int G = g.ngrid;
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = g.inl[j] + w; k < g.inl[j + 1]; k += nw) {
    const int base = lsstart[k], cnt = g.pn_ptr[k + 1] - g.pn_ptr[k];
    for (int t = lane; t < cnt; t += 32) {
      const double* d = fda + 3 * (size_t)(base + t);
      f0 += d[0];
      f1 += d[1];
      f2 += d[2];
    }
  }
  for (int n = threadIdx.x; n < G; n += blockDim.x) {
    const size_t p = (size_t)j * G + n;
    double u = g.ui[p];
    if (u > 0.0 && u < 1.0) {
      double ph = phi[g.cavidx[p]];
      double c = g.grid[n].w * ph * xs[p];
      f0 -= c * g.zi[3 * p];
      f1 -= c * g.zi[3 * p + 1];
      f2 -= c * g.zi[3 * p + 2];
    }
  }
  __shared__ double sh[3][4];
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    f0 += __shfl_xor_sync(0xffffffffu, f0, o);
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
  }
  if (lane == 0) {
    sh[0][w] = f0;
    sh[1][w] = f1;
    sh[2][w] = f2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = fxa[3 * (size_t)j + threadIdx.x];
    for (int ww = 0; ww < nw; ++ww) s += sh[threadIdx.x][ww];
    fx[3 * (size_t)j + threadIdx.x] = fep * s;
  }
}

cudaError_t launch_forces(Launch L, const YlmTables& tb, const DevGeo& g, const double* sigma,
                          const double* s_xi, const double* u_chi, const double* phi,
                          double fep, double* fx, double* fxa, double* fda, double2* fv) {
  if (g.nsph == 0) return cudaSuccess;
  cudaError_t e0 = launch_force_vec(L, tb, g.nsph, sigma, fv);
  if (e0) return e0;
#define CASE(LV)                                                                               \
  case LV:                                                                                     \
    k_forces_a<LV><<<g.nsph, 128, 0, L.st>>>(tb, g, sigma, fv, s_xi, u_chi, phi, fxa, fda);    \
    break;
  switch (tb.lmax) {
    DDC_LMAX_CASES(CASE)
    default:
      return cudaErrorInvalidValue;
  }
#undef CASE
  ++*L.launches;
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  k_forces_b<<<g.nsph, 128, 0, L.st>>>(g, s_xi, phi, fxa, fda, g.lsstart, fep, fx);
  ++*L.launches;
  return cudaGetLastError();
}

// ddmkxi / ddmkzeta (ddcosmo.f90:1758-1806): scale * w_n U_i(n) xi_i(n) at
// the cavity points, xi_grid = basis^T S on the full grid.
__global__ void k_mkxi(int ncav, int G, const int* __restrict__ cavpt,
                       const double4* __restrict__ grid, const double* __restrict__ ui,
                       const double* __restrict__ xig, double scale, double* out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncav) return;
  int p = cavpt[c];
  int n = p % G;
  out[c] = scale * (grid[n].w * ui[p] * xig[p]);
}
cudaError_t launch_mkxi(Launch L, const YlmTables& tb, const DevGeo& g, const double* xi_grid,
                        double scale, double* out) {
  if (g.ncav == 0) return cudaSuccess;
  k_mkxi<<<(g.ncav + 255) / 256, 256, 0, L.st>>>(g.ncav, g.ngrid, g.cavpt, g.grid, g.ui, xi_grid,
                                                  scale, out);
  ++*L.launches;
  return cudaGetLastError();
}

// fx(:,i) -= sum_{cavity points of i} zeta * ef  (main.f90:245-253)
__global__ void k_zeta_contract(int nsph, const int* __restrict__ cavoff,
                                const double* __restrict__ zeta, const double* __restrict__ ef,
                                double* fx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsph) return;
  double a0 = fx[3 * i], a1 = fx[3 * i + 1], a2 = fx[3 * i + 2];
  for (int c = cavoff[i]; c < cavoff[i + 1]; ++c) {
    double z = zeta[c];
    a0 -= z * ef[3 * (size_t)c];
    a1 -= z * ef[3 * (size_t)c + 1];
    a2 -= z * ef[3 * (size_t)c + 2];
  }
  fx[3 * i] = a0;
  fx[3 * i + 1] = a1;
  fx[3 * i + 2] = a2;
}
cudaError_t launch_zeta_efld_contract(Launch L, const DevGeo& g, const double* zeta,
                                      const double* ef, double* fx) {
  if (g.nsph == 0) return cudaSuccess;
  k_zeta_contract<<<(g.nsph + 127) / 128, 128, 0, L.st>>>(g.nsph, g.cavoff, zeta, ef, fx);
  ++*L.launches;
  return cudaGetLastError();
}
// fx(:,i) -= ef(:,i) * q_i  (main.f90:263-265)
__global__ void k_charge_contract(int n, const double* __restrict__ q,
                                  const double* __restrict__ ef, double* fx) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * n) return;
  fx[e] -= ef[e] * q[e / 3];
}
cudaError_t launch_charge_efld_contract(Launch L, int n, const double* q, const double* ef,
                                        double* fx) {
  if (n == 0) return cudaSuccess;
  k_charge_contract<<<(3 * n + 255) / 256, 256, 0, L.st>>>(n, q, ef, fx);
  ++*L.launches;
  return cudaGetLastError();
}
// csph(3,n) and SoA copies of the centres from the packed spheres
__global__ void k_csph_pack(int n, const double4* __restrict__ sph, double* csph, double* sx,
                            double* sy, double* sz) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 s = sph[i];
  csph[3 * i] = s.x;
  csph[3 * i + 1] = s.y;
  csph[3 * i + 2] = s.z;
  sx[i] = s.x;
  sy[i] = s.y;
  sz[i] = s.z;
}
cudaError_t launch_csph_pack(Launch L, int n, const double4* sph, double* csph, double* sx,
                             double* sy, double* sz) {
  if (n == 0) return cudaSuccess;
  k_csph_pack<<<(n + 255) / 256, 256, 0, L.st>>>(n, sph, csph, sx, sy, sz);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP32 operator (mixed precision).  Same work decomposition as the FP64
// kernels; geometry differences are formed in FP64 and rounded once to FP32,
// the recurrences, switch function and accumulations run in FP32.  The
// result is an operator accurate to ~1e-6 relative, used only inside the
// FP64 iterative refinement of the solver (the outer residual is FP64).
// ---------------------------------------------------------------------------
struct AnglesF {
  float c, s, cp, sp;
};
__device__ __forceinline__ AnglesF angles_of_f(float sx, float sy, float sz) {
  AnglesF a;
  a.c = sz;
  a.s = sqrtf(fmaxf(0.f, 1.f - sz * sz));
  if (a.s != 0.f) {
    float r = 1.f / a.s;
    a.cp = sx * r;
    a.sp = sy * r;
  } else {
    a.cp = 1.f;
    a.sp = 0.f;
  }
  return a;
}
__device__ __forceinline__ float fsw_f(float x, float eta, float flow, float a, float b,
                                       float ie5) {
  if (x >= 1.f) return 0.f;
  if (x <= flow) return 1.f;
  float xm = x - 1.f;
  return (xm * xm * (1.f - x)) * ((6.f * x + a) * x + b) * ie5;
}

template <int LMAX>
__device__ __forceinline__ float ylm_dot_f(const YlmTables& tb, const AnglesF& a, float t,
                                           const float2* __restrict__ xs) {
  const float ct = a.c * t, st = a.s * t, t2 = t * t;
  float acc = 0.f, pmm = 1.f;
  float cm = 1.f, sm = 0.f, cmm1 = 1.f, smm1 = 0.f;
#pragma unroll
  for (int m = 0; m <= LMAX; ++m) {
    if (m == 1) {
      cm = a.cp;
      sm = a.sp;
    } else if (m >= 2) {
      float cn = 2.f * a.cp * cm - cmm1, sn = 2.f * a.cp * sm - smm1;
      cmm1 = cm; smm1 = sm; cm = cn; sm = sn;
    }
    float p0 = pmm, p1 = 0.f;
#pragma unroll
    for (int l = m; l <= LMAX; ++l) {
      float P;
      if (l == m) {
        P = p0;
      } else if (l == m + 1) {
        p1 = (float)(2 * m + 1) * ct * p0;
        P = p1;
      } else {
        P = (tb.Af[lmi(l, m)] * ct) * p1 - (tb.Bf[lmi(l, m)] * t2) * p0;
        p0 = p1;
        p1 = P;
      }
      float2 xv = xs[lmi(l, m)];
      float q = (m == 0) ? xv.x : fmaf(cm, xv.x, sm * xv.y);
      acc = fmaf(P, q, acc);
    }
    pmm = -pmm * (float)(2 * m + 1) * st;
  }
  return acc;
}

template <int LMAX>
__global__ void __launch_bounds__(32 * ls_nroles(LMAX)) k_lstarx_f(const YlmTables tb,
                                                                    const DevGeo g,
                                                                    const float* __restrict__ xi,
                                                                    double* y) {
  constexpr int NR = ls_nroles(LMAX);
  constexpr int NT = 32 * NR;
  constexpr int CH = NT;
  constexpr int NVM = ls_max_nvals(LMAX);
  extern __shared__ float shf[];  // [NF][CH]
  const int i = blockIdx.x;
  if (sweep_skip(g.act, i)) return;
  const int role = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double4 ci = g.sph[i];
  const int G = g.ngrid;
  const float eta = (float)tb.eta, flow = 1.f - eta;
  const float fa = 15.f * eta - 12.f, fb = 10.f * eta * eta - 15.f * eta + 6.f;
  const float ie5 = (float)(1.0 / (tb.eta * tb.eta * tb.eta * tb.eta * tb.eta));
  const float iri = (float)(1.0 / ci.w);
  float acc[NVM];
#pragma unroll
  for (int v = 0; v < NVM; ++v) acc[v] = 0.f;
  const int q0 = g.ls_ptr[i], q1 = g.ls_ptr[i + 1];
  for (int c0 = q0; c0 < q1; c0 += CH) {
    const int chunk = min(CH, q1 - c0);
    for (int tt = threadIdx.x; tt < chunk; tt += NT) {
      const int q = c0 + tt;
      const int2 jn = g.ls[q];
      const int j = jn.x, n = jn.y;
      const double4 cj = g.sph[j];
      const float4 gn = g.gridf[n];
      const float rj = (float)cj.w;
      float vx = fmaf(rj, gn.x, (float)(cj.x - ci.x));
      float vy = fmaf(rj, gn.y, (float)(cj.y - ci.y));
      float vz = fmaf(rj, gn.z, (float)(cj.z - ci.z));
      float r2 = vx * vx + vy * vy + vz * vz;
      float rinv = rsqrtf(r2);
      float t = r2 * rinv * iri;
      AnglesF a = angles_of_f(vx * rinv, vy * rinv, vz * rinv);
      const size_t pj = (size_t)j * G + n;
      float chi = fsw_f(t, eta, flow, fa, fb, ie5);
      float f = (float)g.fi[pj];
      float W = f > 1.f ? chi / f : chi;
      const float st = a.s * t;
      float* col = shf + tt;
      col[0] = a.c * t;
      col[CH] = t * t;
      float pmm = gn.w * xi[pj] * W;
      float cm = 1.f, sm = 0.f, cmm1 = 1.f, smm1 = 0.f;
#pragma unroll
      for (int m = 0; m <= LMAX; ++m) {
        if (m == 1) {
          cm = a.cp; sm = a.sp;
        } else if (m >= 2) {
          float cn = 2.f * a.cp * cm - cmm1, sn = 2.f * a.cp * sm - smm1;
          cmm1 = cm; smm1 = sm; cm = cn; sm = sn;
        }
        col[(2 + 3 * m) * CH] = pmm;
        col[(3 + 3 * m) * CH] = cm;
        col[(4 + 3 * m) * CH] = sm;
        pmm = -pmm * (float)(2 * m + 1) * st;
      }
    }
    __syncthreads();
    ls_run_role<LMAX, 0, float>(role, tb, shf, CH, chunk, lane, acc);
    __syncthreads();
  }
  ls_finish_role<LMAX, 0, float>(role, tb, acc, y + (size_t)i * tb.nylm, lane);
}

cudaError_t launch_lstarx_acc_f32(Launch L, const YlmTables& tb, const DevGeo& g,
                                  const float* xi, double* y) {
  if (g.nsph == 0) return cudaSuccess;
  cudaError_t e = cudaSuccess;
#define CASE(LV)                                                                              \
  case LV: {                                                                                  \
    constexpr int NR = ls_nroles(LV);                                                         \
    size_t sm = sizeof(float) * ls_nfields(LV) * 32 * NR;                                     \
    if (sm > 48 * 1024)                                                                       \
      if ((e = cudaFuncSetAttribute(k_lstarx_f<LV>,                                           \
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)))   \
        return e;                                                                             \
    k_lstarx_f<LV><<<g.nsph, 32 * NR, sm, L.st>>>(tb, g, xi, y);                              \
    break;                                                                                    \
  }
  switch (tb.lmax) {
    DDC_LMAX_CASES(CASE)
    default:
      return cudaErrorInvalidValue;
  }
#undef CASE
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fused application of L and L* (lx matvec.f90:94-148 with calcv
// ddcosmo.f90:1671-1746; lstarx matvec.f90:161-235 with adjrhs
// ddcosmo.f90:1301-1384).  Both operators run over the same triples
// (a, n, b): grid point n of sphere a inside sphere b (t < 1).  They share
// the weight W = chi(t) / f_a(n) and the values t^l Y_lm(s), s the unit
// vector from c_b to c_a + r_a s_n:
//   lx     (output a):  pot_a(n) += W sum_lm K_lm t^l Y_lm(s) X_b,lm
//   lstarx (output b):  y_b,lm   -= K_lm w_n xi_a(n) W t^l Y_lm(s)
// Block per sphere b over its gather list (the lstarx layout), in chunks
// of one triple per thread, software pipelined over two shared buffers:
// every thread issues the global loads of its triple of chunk k+1, then the
// role warps (a role owns a set of Legendre columns, below) run the
// normalised recurrence over chunk k and feed each value to
// both contractions (registers accumulate the L* rows, the role's share of
// each triple's lx value goes to shared memory), then the thread turns its
// loaded inputs into chunk k+1's fields (prefix Q_m^m with W folded in,
// cos m phi, sin m phi) in the other buffer.  One barrier per chunk; the
// load latency hides behind the recurrences.  X_b (K-scaled pairs) sits in
// the roles' registers.  The lx value of each triple (the roles' shares
// summed in role order) goes to val[q] in gather-list order; k_lx_gather
// then sums the triples of each point (a, n).  No atomics: the results are
// bit-reproducible.
// ---------------------------------------------------------------------------
// Shared fields of a chunk, in units of Rl with CH triples: a 4-vector
// (ct, t2, c = w_n xi_a(n), q0[0]) per triple, then per column m >= 1 the
// prefix q0[m] (W and t^m folded in) and the pair (cos m phi, sin m phi).
// A role reads a triple with one 4-vector load plus two loads per column
// m >= 1 (column 0 has cos = 1, sin = 0 and its prefix in the 4-vector).
__host__ __device__ constexpr int lxs_nfields(int L) { return 4 + 3 * L; }
__host__ __device__ constexpr int lxs_q0(int CH, int m) { return 4 * CH + 3 * CH * (m - 1); }
__host__ __device__ constexpr int lxs_cs(int CH, int m) { return 4 * CH + 3 * CH * (m - 1) + CH; }
template <class Rl> struct V4T;
template <> struct V4T<float> { typedef float4 T; };
template <> struct V4T<double> { typedef double4 T; };

// Roles of the fused pass: NR warps share the lmax+1 Legendre columns.  Per
// triple a column m costs about 5 (m = 0) or 7 (m > 0) operations for each
// of its lmax+1-m values (recurrence, L* and L contractions) plus a fixed
// part.  FP64 passes keep the pairing m / lmax-m of k_lstarx (lmax/2+1
// roles; their summation order, pinned to the oracle's results at 1e-13,
// stays that of the pairing).  FP32 passes give the columns to the roles
// greedily, the most expensive first, each to the least-loaded role (lowest
// index on ties); a role runs its columns in increasing m and holds them in
// that order in its register arrays.  At lmax 10 the FP32 pass runs four
// roles of about three columns each (128 registers, four blocks of 128
// threads per SM): per triple, each role's fixed cost (header load, loop,
// lx share to shared memory) is paid four times instead of six, 1.25 ms
// per launch at the 20,000-sphere workload against 1.35 ms for six roles
// (paired or greedy alike: the SM is issue-bound, and other blocks fill the
// barrier waits of an uneven role split).
template <class Rl>
__host__ __device__ constexpr int lxs_nroles(int L) {
  return sizeof(Rl) == 4 && L == 10 ? 4 : L / 2 + 1;
}
// blocks per SM the pass is compiled for
template <class Rl>
__host__ __device__ constexpr int lxs_min_blocks(int L) {
  return L > 10 ? 1 : sizeof(Rl) == 8 ? (L <= 8 ? 4 : 2) : L == 10 ? 4 : 3;
}
__host__ __device__ constexpr int lxs_cost(int L, int m) {
  return m == 0 ? 5 * (L + 1) + 4 : 7 * (L + 1 - m) + 4;
}
__host__ __device__ constexpr int lxs_role_of(int L, int NR, int m, bool greedy) {
  if (!greedy) return m <= L - m ? m : L - m;
  int load[DDC_MAX_LMAX + 1] = {};
  int role[DDC_MAX_LMAX + 1] = {};
  bool done[DDC_MAX_LMAX + 1] = {};
  for (int k = 0; k <= L; ++k) {
    int best = -1;
    for (int c = 0; c <= L; ++c)
      if (!done[c] && (best < 0 || lxs_cost(L, c) > lxs_cost(L, best))) best = c;
    int r = 0;
    for (int s = 1; s < NR; ++s)
      if (load[s] < load[r]) r = s;
    done[best] = true;
    load[r] += lxs_cost(L, best);
    role[best] = r;
  }
  return role[m];
}
// offset of column m in its role's register arrays
__host__ __device__ constexpr int lxs_off_of(int L, int NR, int m, bool g) {
  int off = 0;
  for (int c = 0; c < m; ++c)
    if (lxs_role_of(L, NR, c, g) == lxs_role_of(L, NR, m, g)) off += ls_nvals_m(L, c);
  return off;
}
__host__ __device__ constexpr int lxs_role_nvals(int L, int NR, int r, bool g) {
  int n = 0;
  for (int c = 0; c <= L; ++c)
    if (lxs_role_of(L, NR, c, g) == r) n += ls_nvals_m(L, c);
  return n;
}
__host__ __device__ constexpr int lxs_max_nvals(int L, int NR, bool g) {
  int mx = 0;
  for (int r = 0; r < NR; ++r)
    mx = lxs_role_nvals(L, NR, r, g) > mx ? lxs_role_nvals(L, NR, r, g) : mx;
  return mx;
}
__host__ __device__ constexpr int lxs_first_col(int L, int NR, int r, bool g) {
  for (int c = 0; c <= L; ++c)
    if (lxs_role_of(L, NR, c, g) == r) return c;
  return -1;
}

template <class Rl> __device__ __forceinline__ Rl cBn(const YlmTables& tb, int e);
template <> __device__ __forceinline__ double cBn<double>(const YlmTables& tb, int e) { return tb.Bn[e]; }
template <> __device__ __forceinline__ float cBn<float>(const YlmTables& tb, int e) { return tb.Bnf[e]; }

// LONLY: the lx part only (no L* accumulation)
template <int LMAX, int M, int OFF, class Rl, bool LONLY = false>
__device__ __forceinline__ Rl lxs_column(const YlmTables& tb, Rl ct, Rl t2, Rl q0, Rl cm, Rl sm,
                                         Rl c, Rl* acc, const Rl* xr) {
  constexpr int NM = LMAX + 1 - M;
  Rl q1 = 0, dc = 0, ds = 0;
  const Rl cmc = LONLY ? Rl(0) : cm * c, smc = LONLY ? Rl(0) : sm * c;
#pragma unroll
  for (int l = M; l <= LMAX; ++l) {
    Rl Q;
    if (l == M) {
      Q = q0;
    } else if (l == M + 1) {
      q1 = ct * q0;
      Q = q1;
    } else {
      Q = fma(ct, q1, -(cBn<Rl>(tb, lmi(l, M)) * t2) * q0);
      q0 = q1;
      q1 = Q;
    }
    if (M == 0) {
      if (!LONLY) acc[OFF + l] = fma(Q, c, acc[OFF + l]);
      dc = fma(Q, xr[OFF + l], dc);
    } else {
      if (!LONLY) {
        acc[OFF + (l - M)] = fma(Q, cmc, acc[OFF + (l - M)]);
        acc[OFF + NM + (l - M)] = fma(Q, smc, acc[OFF + NM + (l - M)]);
      }
      dc = fma(Q, xr[OFF + (l - M)], dc);
      ds = fma(Q, xr[OFF + NM + (l - M)], ds);
    }
  }
  if (M == 0) return dc;
  return fma(cm, dc, sm * ds);
}

template <int LMAX, int M, int OFF, class Rl>
__device__ __forceinline__ void lxs_load_col(const typename RT<Rl>::V2* __restrict__ xb, Rl* xr) {
  constexpr int NM = LMAX + 1 - M;
#pragma unroll
  for (int l = M; l <= LMAX; ++l) {
    const typename RT<Rl>::V2 v = xb[lmi(l, M)];
    xr[OFF + (l - M)] = v.x;
    if (M > 0) xr[OFF + NM + (l - M)] = v.y;
  }
}

// X_b of role R's columns into its registers
template <int LMAX, int NR, int R, int M, class Rl>
__device__ __forceinline__ void lxs_load_cols(const typename RT<Rl>::V2* xb, Rl* xr) {
  if constexpr (lxs_role_of(LMAX, NR, M, sizeof(Rl) == 4) == R)
    lxs_load_col<LMAX, M, lxs_off_of(LMAX, NR, M, sizeof(Rl) == 4), Rl>(xb, xr);
  if constexpr (M < LMAX) lxs_load_cols<LMAX, NR, R, M + 1, Rl>(xb, xr);
}
template <int LMAX, int NR, int R, class Rl>
__device__ __forceinline__ void lxs_load_role(int role, const typename RT<Rl>::V2* xb, Rl* xr) {
  if (role == R) {
    lxs_load_cols<LMAX, NR, R, 0, Rl>(xb, xr);
    return;
  }
  if constexpr (R + 1 < NR) lxs_load_role<LMAX, NR, R + 1, Rl>(role, xb, xr);
}

// role R's share of triple q: its columns in increasing m, the lx parts
// summed in that order
template <int LMAX, int NR, int R, int M, class Rl, bool LONLY>
__device__ __forceinline__ void lxs_cols(const YlmTables& tb, const Rl* sh, int q,
                                         const typename V4T<Rl>::T& h, Rl* acc, const Rl* xr,
                                         Rl& part) {
  typedef typename RT<Rl>::V2 V2;
  constexpr int CH = 32 * NR;
  if constexpr (lxs_role_of(LMAX, NR, M, sizeof(Rl) == 4) == R) {
    constexpr int OFF = lxs_off_of(LMAX, NR, M, sizeof(Rl) == 4);
    Rl v;
    if constexpr (M == 0) {
      v = lxs_column<LMAX, 0, OFF, Rl, LONLY>(tb, h.x, h.y, h.w, Rl(1), Rl(0), h.z, acc, xr);
    } else {
      const V2 c2 = reinterpret_cast<const V2*>(sh + lxs_cs(CH, M))[q];
      v = lxs_column<LMAX, M, OFF, Rl, LONLY>(tb, h.x, h.y, sh[lxs_q0(CH, M) + q], c2.x, c2.y,
                                              h.z, acc, xr);
    }
    if constexpr (M == lxs_first_col(LMAX, NR, R, sizeof(Rl) == 4)) part = v;
    else part += v;
  }
  if constexpr (M < LMAX) lxs_cols<LMAX, NR, R, M + 1, Rl, LONLY>(tb, sh, q, h, acc, xr, part);
}

// lanes take triples q < count of the chunk's fields sh
template <int LMAX, int NR, int R, class Rl, bool LONLY = false>
__device__ __forceinline__ void lxs_role(const YlmTables& tb, const Rl* sh, int count, int lane,
                                         Rl* acc, const Rl* xr, Rl* lxp) {
  typedef typename V4T<Rl>::T V4;
  constexpr int CH = 32 * NR;
  const V4* hdr = reinterpret_cast<const V4*>(sh);
  for (int q = lane; q < count; q += 32) {
    const V4 h = hdr[q];
    Rl part;
    lxs_cols<LMAX, NR, R, 0, Rl, LONLY>(tb, sh, q, h, acc, xr, part);
    lxp[R * CH + q] = part;
  }
}
template <int LMAX, int NR, int R, class Rl, bool LONLY = false>
__device__ __forceinline__ void lxs_run_role(int role, const YlmTables& tb, const Rl* sh,
                                             int count, int lane, Rl* acc, const Rl* xr,
                                             Rl* lxp) {
  if (role == R) {
    lxs_role<LMAX, NR, R, Rl, LONLY>(tb, sh, count, lane, acc, xr, lxp);
    return;
  }
  if constexpr (R + 1 < NR)
    lxs_run_role<LMAX, NR, R + 1, Rl, LONLY>(role, tb, sh, count, lane, acc, xr, lxp);
}

// the L* rows of role R: lane sums by a fixed shuffle tree, then its columns
// G: the greedy column map (else the pairing); the fused pass's choice by
// default
template <int LMAX, int NR, int R, int M, class Rl, bool GAM, bool G = sizeof(Rl) == 4>
__device__ __forceinline__ void lxs_store_cols(const YlmTables& tb, const Rl* acc, double* yi,
                                               int lane) {
  if constexpr (lxs_role_of(LMAX, NR, M, G) == R)
    ls_store<LMAX, M, lxs_off_of(LMAX, NR, M, G), Rl, GAM>(tb, acc, yi, lane);
  if constexpr (M < LMAX) lxs_store_cols<LMAX, NR, R, M + 1, Rl, GAM, G>(tb, acc, yi, lane);
}
template <int LMAX, int NR, int R, class Rl, bool GAM, bool G = sizeof(Rl) == 4>
__device__ __forceinline__ void lxs_finish_role(int role, const YlmTables& tb, Rl* acc,
                                                double* yi, int lane) {
  if (role == R) {
    constexpr int NV = lxs_role_nvals(LMAX, NR, R, G);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
    }
    lxs_store_cols<LMAX, NR, R, 0, Rl, GAM, G>(tb, acc, yi, lane);
    return;
  }
  if constexpr (R + 1 < NR)
    lxs_finish_role<LMAX, NR, R + 1, Rl, GAM, G>(role, tb, acc, yi, lane);
}

// the inputs of one triple's shared fields, loaded one chunk ahead
template <class Rl>
struct LxsIn {
  double4 ca;
  GP<Rl> gn;
  double f;
  Rl xv;
};
template <class Rl>
__device__ __forceinline__ LxsIn<Rl> lxs_load(const DevGeo& g, const Rl* __restrict__ xi, int q,
                                               int2 an) {
  const size_t pa = (size_t)an.x * g.ngrid + an.y;
  LxsIn<Rl> in;
  in.ca = g.sph[an.x];
  in.gn = grid_pt(g, an.y, (Rl*)nullptr);
  in.f = g.fi[pa];
  in.xv = xi ? xi[pa] : Rl(0);
  return in;
}
// the shared fields of one triple from its inputs (column col of the buffer)
// FP32 path: approximate reciprocal square root and division (about 2 ulp;
// the FP32 operator only has to be accurate to ~1e-6 for the FP64
// refinement); FP64 path: IEEE operations
__device__ __forceinline__ double div_t(double a, double b) { return a / b; }
__device__ __forceinline__ float div_t(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double sin_from_cos(double c) { return sqrt(fmax(0.0, 1.0 - c * c)); }
__device__ __forceinline__ float sin_from_cos(float c) {
  const float u = 1.f - c * c;
  return u > 0.f ? u * rsqrtf(u) : 0.f;
}
// The static geometry of one triple: t cos(theta), t^2, t sin(theta), the
// weight W = chi(t) / f_a(n), cos(phi), sin(phi).
template <class Rl>
struct LxsGeo {
  Rl ct, t2, st, W, cp, sp;
};
template <class Rl>
__device__ __forceinline__ LxsGeo<Rl> lxs_geom(const YlmTables& tb, double4 ca, GP<Rl> gn,
                                               double fd, double4 cb, Rl irb) {
  constexpr bool D = sizeof(Rl) == 8;
  const Rl eta = (Rl)tb.eta, flow = Rl(1) - eta;
  const Rl fa = Rl(15) * eta - Rl(12), fb = Rl(10) * eta * eta - Rl(15) * eta + Rl(6);
  Rl vx, vy, vz;
  if constexpr (D) {
    vx = fma(ca.w, gn.x, ca.x) - cb.x;
    vy = fma(ca.w, gn.y, ca.y) - cb.y;
    vz = fma(ca.w, gn.z, ca.z) - cb.z;
  } else {
    const float ra = (float)ca.w;
    vx = fmaf(ra, gn.x, (float)(ca.x - cb.x));
    vy = fmaf(ra, gn.y, (float)(ca.y - cb.y));
    vz = fmaf(ra, gn.z, (float)(ca.z - cb.z));
  }
  const Rl r2 = vx * vx + vy * vy + vz * vz;
  const Rl rinv = rsqrt_t(r2);
  const Rl t = r2 * rinv * irb;
  const Rl sz = vz * rinv;
  const Rl sth = sin_from_cos(sz);
  LxsGeo<Rl> o;
  o.cp = 1;  // pole: only m = 0 survives
  o.sp = 0;
  if (sth != Rl(0)) {
    const Rl rs = div_t(rinv, sth);
    o.cp = vx * rs;
    o.sp = vy * rs;
  }
  Rl chi;
  if (t >= Rl(1)) chi = 0;
  else if (t <= flow) chi = 1;
  else {
    const Rl xm = t - Rl(1);
    const Rl ie5 = (Rl)(1.0 / (tb.eta * tb.eta * tb.eta * tb.eta * tb.eta));
    chi = (xm * xm * (Rl(1) - t)) * ((Rl(6) * t + fa) * t + fb) * ie5;
  }
  const Rl f = (Rl)fd;
  o.W = f > Rl(1) ? div_t(chi, f) : chi;
  o.st = sth * t;
  o.ct = sz * t;
  o.t2 = t * t;
  return o;
}
// the shared fields of one triple (column tt of the chunk's buffer) from its
// geometry, grid weight and xi_a(n)
template <int LMAX, int NR, class Rl>
__device__ __forceinline__ void lxs_fields(const LxsGeo<Rl>& gm, Rl w, Rl xv, Rl* sh, int tt) {
  constexpr int CH = 32 * NR;
  typedef typename RT<Rl>::V2 V2;
  typedef typename V4T<Rl>::T V4;
  V4 h;
  h.x = gm.ct;
  h.y = gm.t2;
  h.z = w * xv;
  h.w = gm.W;  // q0[0]
  reinterpret_cast<V4*>(sh)[tt] = h;
  const Rl cp = gm.cp, sp = gm.sp, st = gm.st;
  Rl pmm = -gm.W * Rl(1) * st, cm = cp, sm = sp, cmm1 = 1, smm1 = 0;
#pragma unroll
  for (int m = 1; m <= LMAX; ++m) {
    if (m >= 2) {
      const Rl cn = Rl(2) * cp * cm - cmm1, sn = Rl(2) * cp * sm - smm1;
      cmm1 = cm; smm1 = sm; cm = cn; sm = sn;
    }
    sh[lxs_q0(CH, m) + tt] = pmm;
    V2 c2;
    c2.x = cm;
    c2.y = sm;
    reinterpret_cast<V2*>(sh + lxs_cs(CH, m))[tt] = c2;
    pmm = -pmm * Rl(2 * m + 1) * st;
  }
}
template <int LMAX, int NR, class Rl>
__device__ __forceinline__ void lxs_fields(const YlmTables& tb, const LxsIn<Rl>& in, double4 cb,
                                           Rl irb, Rl* sh, int tt) {
  lxs_fields<LMAX, NR, Rl>(lxs_geom<Rl>(tb, in.ca, in.gn, in.f, cb, irb), in.gn.w, in.xv, sh, tt);
}
// the geometry precomputed at ddinit (DevGeo::tgeo4/tgeo2 in FP32,
// tgeo4d/tgeo2d in FP64)
template <class Rl>
struct LxsInP {
  typename V4T<Rl>::T g4;  // ct, t2, st, W
  typename RT<Rl>::V2 g2;  // cp, sp
  Rl w, xv;
};
__device__ __forceinline__ float4 tgeo4_of(const DevGeo& g, int q, float*) { return g.tgeo4[q]; }
__device__ __forceinline__ double4 tgeo4_of(const DevGeo& g, int q, double*) { return g.tgeo4d[q]; }
__device__ __forceinline__ float2 tgeo2_of(const DevGeo& g, int q, float*) { return g.tgeo2[q]; }
__device__ __forceinline__ double2 tgeo2_of(const DevGeo& g, int q, double*) { return g.tgeo2d[q]; }
template <class Rl>
__device__ __forceinline__ LxsInP<Rl> lxs_load_pre(const DevGeo& g, const Rl* __restrict__ xi,
                                                   int q, int2 an) {
  LxsInP<Rl> in;
  in.g4 = tgeo4_of(g, q, (Rl*)nullptr);
  in.g2 = tgeo2_of(g, q, (Rl*)nullptr);
  in.w = grid_pt(g, an.y, (Rl*)nullptr).w;
  in.xv = xi ? xi[(size_t)an.x * g.ngrid + an.y] : Rl(0);
  return in;
}
template <int LMAX, int NR, class Rl>
__device__ __forceinline__ void lxs_fields_pre(const LxsInP<Rl>& in, Rl* sh, int tt) {
  LxsGeo<Rl> gm;
  gm.ct = in.g4.x;
  gm.t2 = in.g4.y;
  gm.st = in.g4.z;
  gm.W = in.g4.w;
  gm.cp = in.g2.x;
  gm.sp = in.g2.y;
  lxs_fields<LMAX, NR, Rl>(gm, in.w, in.xv, sh, tt);
}
// the geometry of every triple, block per sphere b over its gather list
template <class Rl>
__global__ void k_lxs_geo(const YlmTables tb, const DevGeo g, typename V4T<Rl>::T* tg4,
                          typename RT<Rl>::V2* tg2) {
  const int b = blockIdx.x;
  const double4 cb = g.sph[b];
  const Rl irb = (Rl)(1.0 / cb.w);
  for (int q = g.ls_ptr[b] + threadIdx.x; q < g.ls_ptr[b + 1]; q += blockDim.x) {
    const int2 an = g.ls[q];
    const LxsGeo<Rl> gm = lxs_geom<Rl>(tb, g.sph[an.x], grid_pt(g, an.y, (Rl*)nullptr),
                                       g.fi[(size_t)an.x * g.ngrid + an.y], cb, irb);
    tg4[q].x = gm.ct;
    tg4[q].y = gm.t2;
    tg4[q].z = gm.st;
    tg4[q].w = gm.W;
    tg2[q].x = gm.cp;
    tg2[q].y = gm.sp;
  }
}
cudaError_t launch_lxs_geo(Launch L, const YlmTables& tb, const DevGeo& g, float4* tg4,
                           float2* tg2) {
  if (g.nsph == 0) return cudaSuccess;
  k_lxs_geo<float><<<g.nsph, 128, 0, L.st>>>(tb, g, tg4, tg2);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_lxs_geo_f64(Launch L, const YlmTables& tb, const DevGeo& g, double4* tg4,
                               double2* tg2) {
  if (g.nsph == 0) return cudaSuccess;
  k_lxs_geo<double><<<g.nsph, 128, 0, L.st>>>(tb, g, tg4, tg2);
  ++*L.launches;
  return cudaGetLastError();
}

// FP32 chunks are double-buffered (software pipeline); FP64 chunks use one
// buffer so that two blocks fit in shared memory
template <class Rl> __host__ __device__ constexpr bool lxs_piped() { return sizeof(Rl) == 4; }
// Blocks per SM: lxs_min_blocks (FP32 at lmax 10: four of 128 threads, at
// most 128 registers; other FP32 cases three; FP64 up to lmax 8 four, at
// most 128 registers: 253 against 282 ms for the 256-globule batch solve at
// lmax 6 with two; FP64 at lmax 9-10 two, at most 168)
// MODE 0: L x (val) and L* xi (y) together; 1: L x only (xi, y unused);
// 2: L x only with the weight chi(t) in place of chi(t)/f_a(n) (the u_chi sum
// of the forces, on-the-fly geometry only)
template <int LMAX, class Rl, bool PRE = false, int MODE = 0>
__global__ void __launch_bounds__(32 * lxs_nroles<Rl>(LMAX), lxs_min_blocks<Rl>(LMAX))
    k_lxs(const YlmTables tb, const DevGeo g, const typename RT<Rl>::V2* __restrict__ XK,
          const Rl* __restrict__ xi, Rl* __restrict__ val, double* __restrict__ y) {
  static_assert(!(PRE && MODE == 2), "chi-only weights need the on-the-fly geometry");
  constexpr bool LONLY = MODE != 0;
  constexpr int NR = lxs_nroles<Rl>(LMAX);
  constexpr int CH = 32 * NR;  // triples per chunk = threads per block
  constexpr int NF = lxs_nfields(LMAX);
  constexpr int NVM = lxs_max_nvals(LMAX, NR, sizeof(Rl) == 4);
  constexpr int NLM = (LMAX + 1) * (LMAX + 2) / 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int NBUF = lxs_piped<Rl>() ? 2 : 1;
  Rl* fld = reinterpret_cast<Rl*>(smraw);  // [NBUF][NF][CH]
  Rl* lxp = fld + NBUF * NF * CH;          // [NBUF][NR][CH]
  const int b = blockIdx.x, tid = threadIdx.x;
  if (sweep_skip(g.act, b)) return;
  const int role = tid >> 5, lane = tid & 31;
  const int q0 = g.ls_ptr[b], q1 = g.ls_ptr[b + 1];
  const int nch = (q1 - q0 + CH - 1) / CH;
  const double4 cb = g.sph[b];
  const Rl irb = (Rl)(1.0 / cb.w);
  Rl acc[NVM], xr[NVM];
#pragma unroll
  for (int v = 0; v < NVM; ++v) acc[v] = xr[v] = 0;
  lxs_load_role<LMAX, NR, 0, Rl>(role, XK + (size_t)b * NLM, xr);
  // with the geometry precomputed at ddinit only xi_a(n) and the grid weight
  // are read per triple besides the two geometry vectors
  typedef typename std::conditional<PRE, LxsInP<Rl>, LxsIn<Rl>>::type In;
  // an: the triple's gather-list entry (a, n), loaded a chunk earlier than
  // the inputs that depend on it
  auto load = [&](int q, int2 an) -> In {
    if constexpr (PRE) {
      return lxs_load_pre<Rl>(g, LONLY ? nullptr : xi, q, an);
    } else {
      In in = lxs_load<Rl>(g, LONLY ? nullptr : xi, q, an);
      if constexpr (MODE == 2) in.f = 1.0;  // W = chi(t)
      return in;
    }
  };
  auto fields = [&](const In& in, Rl* buf) {
    if constexpr (PRE) lxs_fields_pre<LMAX, NR, Rl>(in, buf, tid);
    else lxs_fields<LMAX, NR, Rl>(tb, in, cb, irb, buf, tid);
  };
  if constexpr (!lxs_piped<Rl>()) {
    // FP64: one buffer (two blocks per SM fit), two barriers per chunk; the
    // inputs of chunk k+1 are loaded while the roles work on chunk k
    In cur;
    int2 an1 = make_int2(0, 0);
    if (nch > 0 && tid < min(CH, q1 - q0)) cur = load(q0 + tid, g.ls[q0 + tid]);
    if (nch > 1 && tid < min(CH, q1 - q0 - CH)) an1 = g.ls[q0 + CH + tid];
    for (int k = 0; k < nch; ++k) {
      const int c0 = q0 + k * CH, cnt = min(CH, q1 - c0);
      if (tid < cnt) fields(cur, fld);
      __syncthreads();
      const int n1 = k + 1 < nch ? min(CH, q1 - c0 - CH) : 0;
      const int n2 = k + 2 < nch ? min(CH, q1 - c0 - 2 * CH) : 0;
      if (tid < n1) cur = load(c0 + CH + tid, an1);
      if (tid < n2) an1 = g.ls[c0 + 2 * CH + tid];
      lxs_run_role<LMAX, NR, 0, Rl, LONLY>(role, tb, fld, cnt, lane, acc, xr, lxp);
      __syncthreads();
      if (tid < cnt) {
        Rl sv = lxp[tid];
#pragma unroll
        for (int r = 1; r < NR; ++r) sv += lxp[r * CH + tid];
        val[c0 + tid] = sv;
      }
    }
    if constexpr (!LONLY)
      lxs_finish_role<LMAX, NR, 0, Rl, true>(role, tb, acc, y + (size_t)b * tb.nylm, lane);
    return;
  }
  if constexpr (PRE && lxs_piped<Rl>()) {
    // FP32 with the geometry precomputed at ddinit: each thread copies its
    // triple's two geometry vectors (24 bytes) to its own shared slot with
    // cp.async two chunks ahead of their use (two chunks of role work cover
    // the latency, and no registers hold them meanwhile; a thread reads only
    // the slot it wrote, after its own wait_group).  The grid weight and
    // xi_a(n) come through registers one chunk ahead, the gather-list entry
    // that addresses them two chunks ahead.  (xi_a(n) by cp.async as well
    // was slower: the copy's issue waits for its gather-list entry.)
    typename V4T<Rl>::T* gs4 = reinterpret_cast<typename V4T<Rl>::T*>(lxp + NBUF * NR * CH);
    typename RT<Rl>::V2* gs2 = reinterpret_cast<typename RT<Rl>::V2*>(gs4 + 2 * CH);
    auto geo_copy = [&](int k) {  // chunk k's geometry into stage k & 1
      const int q = q0 + k * CH + tid;
      if (k < nch && q < q1) {
        cp_async16(gs4 + (k & 1) * CH + tid, g.tgeo4 + q);
        cp_async8(gs2 + (k & 1) * CH + tid, g.tgeo2 + q, true);
      }
      cp_async_commit();
    };
    auto wx = [&](int2 an, Rl& w, Rl& xv) {
      w = grid_pt(g, an.y, (Rl*)nullptr).w;
      xv = LONLY ? Rl(0) : xi[(size_t)an.x * g.ngrid + an.y];
    };
    auto fields_at = [&](int k, Rl w, Rl xv) {
      LxsInP<Rl> in;
      in.g4 = gs4[(k & 1) * CH + tid];
      in.g2 = gs2[(k & 1) * CH + tid];
      in.w = w;
      in.xv = xv;
      lxs_fields_pre<LMAX, NR, Rl>(in, fld + (k & 1) * NF * CH, tid);
    };
    geo_copy(0);
    geo_copy(1);
    Rl w1 = 0, xv1 = 0;
    int2 an1 = make_int2(0, 0);
    if (nch > 0 && tid < min(CH, q1 - q0)) wx(g.ls[q0 + tid], w1, xv1);
    if (nch > 1 && tid < min(CH, q1 - q0 - CH)) an1 = g.ls[q0 + CH + tid];
    cp_async_wait<1>();
    if (nch > 0 && tid < min(CH, q1 - q0)) fields_at(0, w1, xv1);
    __syncthreads();
    for (int k = 0; k < nch; ++k) {
      const int c0 = q0 + k * CH, cnt = min(CH, q1 - c0);
      const int n1 = k + 1 < nch ? min(CH, q1 - c0 - CH) : 0;
      const int n2 = k + 2 < nch ? min(CH, q1 - c0 - 2 * CH) : 0;
      geo_copy(k + 2);
      if (tid < n1) wx(an1, w1, xv1);
      int2 an2 = make_int2(0, 0);
      if (tid < n2) an2 = g.ls[c0 + 2 * CH + tid];
      lxs_run_role<LMAX, NR, 0, Rl, LONLY>(role, tb, fld + (k & 1) * NF * CH, cnt, lane, acc,
                                           xr, lxp + (k & 1) * NR * CH);
      cp_async_wait<1>();  // chunk k+1's copies done (chunk k+2's may be in flight)
      if (tid < n1) fields_at(k + 1, w1, xv1);
      __syncthreads();
      if (tid < cnt) {
        const Rl* lp = lxp + (k & 1) * NR * CH;
        Rl sv = lp[tid];
#pragma unroll
        for (int r = 1; r < NR; ++r) sv += lp[r * CH + tid];
        val[c0 + tid] = sv;
      }
      an1 = an2;
    }
    cp_async_wait<0>();
    if constexpr (!LONLY)
      lxs_finish_role<LMAX, NR, 0, Rl, true>(role, tb, acc, y + (size_t)b * tb.nylm, lane);
    return;
  }
  if (nch > 0 && tid < min(CH, q1 - q0)) fields(load(q0 + tid, g.ls[q0 + tid]), fld);
  int2 an1 = make_int2(0, 0);
  if (nch > 1 && tid < min(CH, q1 - q0 - CH)) an1 = g.ls[q0 + CH + tid];
  __syncthreads();
  // chunk k: loads of chunk k+1 (and the gather-list entries of chunk k+2)
  // in flight while the roles work on chunk k, then chunk k+1's fields go to
  // the other buffer; one barrier per chunk
  for (int k = 0; k < nch; ++k) {
    const int c0 = q0 + k * CH, cnt = min(CH, q1 - c0);
    const int n1 = k + 1 < nch ? min(CH, q1 - c0 - CH) : 0;
    const int n2 = k + 2 < nch ? min(CH, q1 - c0 - 2 * CH) : 0;
    In nxt;
    if (tid < n1) nxt = load(c0 + CH + tid, an1);
    int2 an2 = make_int2(0, 0);
    if (tid < n2) an2 = g.ls[c0 + 2 * CH + tid];
    lxs_run_role<LMAX, NR, 0, Rl, LONLY>(role, tb, fld + (k & 1) * NF * CH, cnt, lane, acc, xr,
                                     lxp + (k & 1) * NR * CH);
    if (tid < n1) fields(nxt, fld + ((k + 1) & 1) * NF * CH);
    __syncthreads();
    // lx values of chunk k: the roles' shares in role order (buffer k&1 of
    // lxp is next written two chunks on, after the next barrier)
    if (tid < cnt) {
      const Rl* lp = lxp + (k & 1) * NR * CH;
      Rl sv = lp[tid];
#pragma unroll
      for (int r = 1; r < NR; ++r) sv += lp[r * CH + tid];
      val[c0 + tid] = sv;
    }
    an1 = an2;
  }
  if constexpr (!LONLY)
    lxs_finish_role<LMAX, NR, 0, Rl, true>(role, tb, acc, y + (size_t)b * tb.nylm, lane);
}

// pot_a(n) = sum over a's CSR pairs (a, b), in CSR order, of the lx values
// of the triples (a, n, b), read from b's gather list at the pair's block
// (lsstart).  Warp per sphere a, with a private shared row of ngrid values
// and the pairs' bounds staged in shared memory: lanes take the pair's
// points (distinct within a pair, so no two lanes touch one entry), four
// strided loads per lane, and the next pair's first loads are issued before
// the current pair's adds; a __syncwarp between pairs orders the updates of
// a point by its pairs.  No block barriers (each warp runs its sphere from
// start to end) and no atomics: a fixed summation order.
constexpr int kGatherWarps = 4;  // spheres per block
template <class Rl>
__global__ void __launch_bounds__(32 * kGatherWarps)
    k_lx_gather(const DevGeo g, const Rl* __restrict__ val, Rl* pot, int ldp) {
  constexpr int U = 4;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int G = g.ngrid;
  const int mb = (g.maxnb + 3) & ~3;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = blockIdx.x * kGatherWarps + w;
  // warp-uniform; the kernel has no block barriers
  if (a >= g.nsph || sweep_skip(g.act, a)) return;
  // per warp: pst[mb + 4] (pn_ptr of the pairs), dl[mb] (lsstart - pn_ptr),
  // then the row (16-byte aligned: mb is a multiple of four)
  int* pst = reinterpret_cast<int*>(smraw) + (size_t)w * (2 * mb + 4);
  int* dl = pst + mb + 4;
  Rl* row = reinterpret_cast<Rl*>(reinterpret_cast<int*>(smraw) + kGatherWarps * (2 * mb + 4)) +
            (size_t)w * G;
  const int k0 = g.inl[a], nn = g.inl[a + 1] - k0;
  for (int k = lane; k <= nn; k += 32) pst[k] = g.pn_ptr[k0 + k];
  for (int k = lane; k < nn; k += 32) dl[k] = g.lsstart[k0 + k] - g.pn_ptr[k0 + k];
  for (int n = lane; n < G; n += 32) row[n] = Rl(0);
  __syncwarp();
  auto load = [&](int base, int q1, int d, int* n, Rl* v) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = base + 32 * u;
      n[u] = q < q1 ? (int)g.pn[q] : -1;
      v[u] = q < q1 ? val[q + d] : Rl(0);
    }
  };
  auto add = [&](const int* n, const Rl* v) {
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (n[u] >= 0) row[n[u]] += v[u];
  };
  int cn[U];
  Rl cv[U];
  if (nn > 0) load(pst[0] + lane, pst[1], dl[0], cn, cv);
  for (int p = 0; p < nn; ++p) {
    const int q0 = pst[p], q1 = pst[p + 1], d = dl[p];
    int nn1[U];
    Rl nv1[U];
    const bool more = p + 1 < nn;
    if (more) load(pst[p + 1] + lane, pst[p + 2], dl[p + 1], nn1, nv1);
    add(cn, cv);
    for (int base = q0 + lane + 32 * U; base < q1; base += 32 * U) {
      int n2[U];
      Rl v2[U];
      load(base, q1, d, n2, v2);
      add(n2, v2);
    }
    __syncwarp();
    if (more) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        cn[u] = nn1[u];
        cv[u] = nv1[u];
      }
    }
  }
  for (int n = lane; n < G; n += 32) pot[(size_t)a * ldp + n] = row[n];
}

template <class Rl, int MODE>
static cudaError_t lxs_launch(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                              const Rl* xi, void* xk, Rl* val, double* y) {
  if (g.nsph == 0) return cudaSuccess;
  typedef typename RT<Rl>::V2 V2;
  const long long nk = (long long)g.nsph * ((tb.lmax + 1) * (tb.lmax + 2) / 2);
  if (nk >= INT_MAX) return cudaErrorInvalidValue;
  V2* XK = static_cast<V2*>(xk);
  k_xk<Rl, true><<<(unsigned)((nk + 255) / 256), 256, 0, L.st>>>(tb, g.nsph, X, XK);
  ++*L.launches;
  cudaError_t e = cudaGetLastError();
  if (e) return e;
#define CASE(LV)                                                                              \
  case LV: {                                                                                  \
    constexpr int NR = lxs_nroles<Rl>(LV);                                                    \
    const bool pre = MODE != 2 && (sizeof(Rl) == 4 ? g.tgeo4 != nullptr : g.tgeo4d != nullptr); \
    const size_t sm = sizeof(Rl) * (lxs_piped<Rl>() ? 2 : 1) * (lxs_nfields(LV) + NR) * 32 * NR + \
                      (pre && lxs_piped<Rl>() ? 2 * 32 * NR * 6 * sizeof(Rl) : 0);             \
    auto kfn = pre ? k_lxs<LV, Rl, MODE != 2, MODE> : k_lxs<LV, Rl, false, MODE>;             \
    if (sm > 48 * 1024) {                                                                     \
      if ((e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                    (int)sm)))                                                \
        return e;                                                                             \
      if ((e = cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout,      \
                                    100)))                                                    \
        return e;                                                                             \
    }                                                                                         \
    kfn<<<g.nsph, 32 * NR, sm, L.st>>>(tb, g, XK, xi, val, y);                                \
    break;                                                                                    \
  }
  switch (tb.lmax) {
    DDC_LMAX_CASES(CASE)
    default:
      return cudaErrorInvalidValue;
  }
#undef CASE
  ++*L.launches;
  return cudaGetLastError();
}
template <class Rl>
static cudaError_t gather_launch(Launch L, const DevGeo& g, const Rl* val, Rl* pot, int ldp) {
  if (g.nsph == 0) return cudaSuccess;
  const int mb = (g.maxnb + 3) & ~3;
  const size_t sm = kGatherWarps * (sizeof(int) * (2 * mb + 4) + sizeof(Rl) * g.ngrid);
  cudaError_t e;
  if (sm > 48 * 1024)
    if ((e = cudaFuncSetAttribute(k_lx_gather<Rl>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm)))
      return e;
  k_lx_gather<Rl><<<(g.nsph + kGatherWarps - 1) / kGatherWarps, 32 * kGatherWarps, sm, L.st>>>(
      g, val, pot, ldp);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_lxs(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                       const double* xi, void* xk, double* val, double* y) {
  return lxs_launch<double, 0>(L, tb, g, X, xi, xk, val, y);
}
cudaError_t launch_lxs_f32(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                           const float* xi, void* xk, float* val, double* y) {
  return lxs_launch<float, 0>(L, tb, g, X, xi, xk, val, y);
}
cudaError_t launch_lx_vals(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                           void* xk, double* val, bool chi_only) {
  return chi_only ? lxs_launch<double, 2>(L, tb, g, X, nullptr, xk, val, nullptr)
                  : lxs_launch<double, 1>(L, tb, g, X, nullptr, xk, val, nullptr);
}
cudaError_t launch_lx_vals_f32(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                               void* xk, float* val) {
  return lxs_launch<float, 1>(L, tb, g, X, nullptr, xk, val, nullptr);
}
cudaError_t launch_lx_gather(Launch L, const DevGeo& g, const double* val, double* pot) {
  return gather_launch<double>(L, g, val, pot, g.ngrid);
}
cudaError_t launch_lx_gather_f32(Launch L, const DevGeo& g, const float* val, float* pot,
                                 int ldp) {
  return gather_launch<float>(L, g, val, pot, ldp);
}

__global__ void k_to_float(long long n, const double* __restrict__ x, float* y) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) y[e] = (float)x[e];
}
cudaError_t launch_to_float(Launch L, long long n, const double* x, float* y) {
  if (n == 0) return cudaSuccess;
  k_to_float<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(n, x, y);
  ++*L.launches;
  return cudaGetLastError();
}
// FP64 residual of the full operator L = D + O at x (y = O x):
//   r = rhs - y - x / facl,  d = facl * r  (the Jacobi increment at x)
// plus the partial sum of the increment's H-norm (hnorm, matvec.f90:281-323)
__global__ void __launch_bounds__(256) k_residual(const YlmTables tb, long long n,
                                                  const double* __restrict__ rhs,
                                                  const double* __restrict__ y,
                                                  const double* __restrict__ x, double* r,
                                                  double* d, double* partials) {
  double acc = 0.0;
  for (LmWalk w(tb.nylm); w.q < n; w.next()) {
    const long long q = w.q;
    int l = l_of(w.lm);
    double fl = tb.facl[l];
    double rv = rhs[q] - y[q] - x[q] / fl;
    double dv = fl * rv;
    r[q] = rv;
    d[q] = dv;
    acc = fma(dv * dv, 1.0 / (1.0 + l), acc);
  }
  double v[1] = {acc};
  block_sum_store<1>(v, 1, partials);
}
cudaError_t launch_residual(Launch L, const YlmTables& tb, long long n, const double* rhs,
                            const double* y, const double* x, double* r, double* d,
                            double* partials, int nblk) {
  k_residual<<<nblk, 256, 0, L.st>>>(tb, n, rhs, y, x, r, d, partials);
  ++*L.launches;
  return cudaGetLastError();
}
__global__ void k_axpy(long long n, double a, const double* __restrict__ x, double* y) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) y[e] = fma(a, x[e], y[e]);
}
cudaError_t launch_axpy(Launch L, long long n, double a, const double* x, double* y) {
  if (n == 0) return cudaSuccess;
  k_axpy<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(n, a, x, y);
  ++*L.launches;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batched solves: many molecules concatenated into one system.  The
// operators act per sphere and need no change; the Jacobi/DIIS driver
// (jacobi_diis.f90) runs per molecule over element chunks (below).
// ---------------------------------------------------------------------------
// Gauss-Jordan with full pivoting (gjinv, jacobi_diis.f90:272-360), one warp,
// lane j owns row j.  a is n x n column-major in shared memory, b the rhs.
// Pivot: the first maximum of |a| over free rows/columns in the reference's
// scan order (rows outer, columns inner).  Returns false when singular.
__device__ bool gjinv_warp(int n, double* a, double* b, int* piv) {
  const int lane = threadIdx.x & 31;
  if (lane < n) piv[lane] = 0;
  __syncwarp();
  for (int i = 0; i < n; ++i) {
    double bv = 0.0;
    int bk = -1;
    if (lane < n && piv[lane] != 1) {
      for (int k = 0; k < n; ++k)
        if (piv[k] == 0) {
          double v = fabs(a[k * n + lane]);
          if (v > bv) {
            bv = v;
            bk = k;
          }
        }
    }
    int bj = bk >= 0 ? lane : 1 << 30;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      int oj = __shfl_xor_sync(0xffffffffu, bj, o);
      int ok = __shfl_xor_sync(0xffffffffu, bk, o);
      if (ov > bv || (ov == bv && oj < bj)) {
        bv = ov;
        bj = oj;
        bk = ok;
      }
    }
    if (bk < 0) return false;  // no non-zero free entry
    const int irow = bj, icol = bk;
    __syncwarp();
    if (lane == 0) piv[icol] += 1;
    __syncwarp();
    if (piv[icol] > 1) return false;
    if (irow != icol) {
      for (int k = lane; k < n; k += 32) {
        double t = a[k * n + irow];
        a[k * n + irow] = a[k * n + icol];
        a[k * n + icol] = t;
      }
      if (lane == 0) {
        double t = b[irow];
        b[irow] = b[icol];
        b[icol] = t;
      }
    }
    __syncwarp();
    const double piv_v = a[icol * n + icol];
    if (piv_v == 0.0) return false;
    const double pinv = 1.0 / piv_v;
    __syncwarp();
    if (lane == 0) a[icol * n + icol] = 1.0;
    __syncwarp();
    for (int k = lane; k < n; k += 32) a[k * n + icol] *= pinv;
    if (lane == 0) b[icol] *= pinv;
    __syncwarp();
    double dum = 0.0;
    if (lane < n && lane != icol) dum = a[icol * n + lane];
    __syncwarp();
    if (lane < n && lane != icol) {
      a[icol * n + lane] = 0.0;
      for (int k = 0; k < n; ++k) a[k * n + lane] -= a[k * n + icol] * dum;
      b[lane] -= b[icol] * dum;
    }
    __syncwarp();
  }
  return true;
}

// The per-molecule Jacobi/DIIS step runs over element chunks of kBChunk
// consecutive elements (a molecule owns one or more chunks), so that a
// large molecule's vectors are read by many blocks at once.  Two kernels:
// k_batch_gram forms the Jacobi iterate, the increment and the chunk's Gram
// partials, and the molecule's last chunk to finish sums the partials in
// chunk order, updates the bordered matrix and solves it (one warp);
// k_batch_extrap forms the extrapolated iterate and the chunk's part of the
// increment norm, and the molecule's last chunk sets its norm, iteration
// count and status.  The history reads are spread over the whole device.
constexpr int kBChunk = kBatchChunk;
static_assert(kBChunk % (kSolU * kSolT) == 0 && kBChunk % (32 * 16) == 0, "chunk tiling");

// Logical-to-physical history slots of molecule k for this step: after
// `nmat` reaches ndiis the ten oldest are dropped (jacobi_diis.f90:196-205).
__device__ __forceinline__ int batch_hist_perm(const BatchState& bs, int k, int* pm) {
  const int nd = bs.ndiis, nm_old = bs.nmat[k];
  const bool shift = nm_old >= nd;
  const int* sl = bs.slot + (size_t)k * nd;
  for (int j = threadIdx.x; j < nd; j += blockDim.x) pm[j] = shift ? sl[(j + 10) % nd] : sl[j];
  return shift ? nm_old - 10 : nm_old;
}

// Last arriving chunk of molecule k (the counter is reset for the next
// kernel).  Every block of the molecule calls it after writing its partials.
__device__ __forceinline__ bool batch_last_chunk(const BatchState& bs, int k) {
  __shared__ unsigned s_last;
  __threadfence();
  __syncthreads();
  const unsigned nc = (unsigned)(bs.cfirst[k + 1] - bs.cfirst[k]);
  if (threadIdx.x == 0) {
    s_last = atomicAdd(bs.cnt + k, 1u) == nc - 1 ? 1u : 0u;
    if (s_last) bs.cnt[k] = 0u;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last != 0;
}

// Sums entries [0, nv) of molecule k's chunk partials in chunk order.
__device__ __forceinline__ void batch_sum_parts(const BatchState& bs, int k, int nv,
                                                double* out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int c0 = bs.cfirst[k], c1 = bs.cfirst[k + 1];
  for (int h = w; h < nv; h += nw) {
    double v = 0.0;
    for (int c = c0 + lane; c < c1; c += 32) v += __ldcg(bs.part + (size_t)c * (kMaxHist + 1) + h);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[h] = v;
  }
  __syncthreads();
}

template <class H>
__global__ void __launch_bounds__(kSolT) k_batch_gram(const YlmTables tb, BatchState bs,
                                                      const double* __restrict__ rhs,
                                                      const double* __restrict__ y,
                                                      const double* __restrict__ x) {
  constexpr int U = kBChunk / kSolT;
  constexpr int NW = kSolT / 32;
  constexpr int KS = (kMaxHist + NW - 1) / NW;
  constexpr int HL = 16;
  const int c = blockIdx.x, k = bs.cmol[c];
  if (bs.status[k] != 0) return;
  __shared__ int pm[kMaxHist];
  __shared__ double es[kBChunk];
  __shared__ double red[kMaxHist + 1 + NW];
  __shared__ double row[kMaxHist + 1];
  const int nm = batch_hist_perm(bs, k, pm), nh = nm - 1;
  __syncthreads();
  const int nylm = tb.nylm, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long N = bs.n_total;
  const long long b0 = (long long)bs.off[k] * nylm + (long long)(c - bs.cfirst[k]) * kBChunk;
  const int cnt = (int)min((long long)kBChunk, (long long)bs.off[k + 1] * nylm - b0);
  H* xnew = static_cast<H*>(bs.hx) + (size_t)pm[nm - 1] * N;
  H* enew = static_cast<H*>(bs.he) + (size_t)pm[nm - 1] * N;
  double ee = 0.0;
  {
    const int dt = kSolT % nylm;
    int lm = (int)((b0 + threadIdx.x) % nylm);
    double rv[U], yv[U], xv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = threadIdx.x + u * kSolT;
      rv[u] = j < cnt ? rhs[b0 + j] : 0.0;
      yv[u] = j < cnt ? y[b0 + j] : 0.0;
      xv[u] = j < cnt ? x[b0 + j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = threadIdx.x + u * kSolT;
      double ev = 0.0;
      if (j < cnt) {
        const double xn = tb.facl[l_of(lm)] * (rv[u] - yv[u]);
        const H eh = (H)(xn - xv[u]);
        ev = (double)eh;
        xnew[b0 + j] = (H)xn;
        enew[b0 + j] = eh;
      }
      es[j] = ev;
      ee = fma(ev, ev, ee);
      lm = lm_add(lm, dt, nylm);
    }
  }
  __syncthreads();
  double d[KS];
#pragma unroll
  for (int s = 0; s < KS; ++s) {
    d[s] = 0.0;
    const int kk = w + NW * s;
    if (kk < nh) {
      const H* hk = static_cast<const H*>(bs.he) + (size_t)pm[kk] * N + b0;
      for (int j0 = 0; j0 < kBChunk; j0 += 32 * HL) {
        H hv[HL];
#pragma unroll
        for (int u = 0; u < HL; ++u) {
          const int j = j0 + u * 32 + lane;
          hv[u] = j < cnt ? hk[j] : H(0);
        }
#pragma unroll
        for (int u = 0; u < HL; ++u) d[s] = fma(es[j0 + u * 32 + lane], (double)hv[u], d[s]);
      }
    }
  }
#pragma unroll
  for (int s = 0; s < KS; ++s) {
    double v = d[s];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int kk = w + NW * s;
    if (lane == 0 && kk < nh) red[kk] = v;
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) ee += __shfl_xor_sync(0xffffffffu, ee, o);
  if (lane == 0) red[kMaxHist + 1 + w] = ee;
  __syncthreads();
  double* part = bs.part + (size_t)c * (kMaxHist + 1);
  if (threadIdx.x < nh) {
    part[threadIdx.x] = red[threadIdx.x];
  } else if (threadIdx.x == nh) {
    double t = 0.0;
    for (int ww = 0; ww < NW; ++ww) t += red[kMaxHist + 1 + ww];
    part[nh] = t;
  }
  if (!batch_last_chunk(bs, k)) return;
  batch_sum_parts(bs, k, nh + 1, row);
  if (threadIdx.x >= 32) return;
  // bordered Gram matrix (makeb, jacobi_diis.f90:232-270) and its solve
  __shared__ double ga[(kMaxHist + 1) * (kMaxHist + 1)], gb[kMaxHist + 1];
  __shared__ int gpiv[kMaxHist + 1];
  const int nd = bs.ndiis, lenb = nd + 1, nm_old = bs.nmat[k];
  double* B = bs.B + (size_t)k * lenb * lenb;
  auto Bm = [&](int j, int kk) -> double& { return B[(size_t)(kk - 1) * lenb + (j - 1)]; };
  if (threadIdx.x == 0) {
    if (nm_old >= nd) {
      for (int j = 2; j <= nm_old - 10; ++j)
        for (int kk = 2; kk <= nm_old - 10; ++kk) Bm(j, kk) = Bm(j + 10, kk + 10);
    }
    if (nm == 1) {
      Bm(1, 1) = 0.0;
      Bm(1, 2) = 1.0;
      Bm(2, 1) = 1.0;
      Bm(2, 2) = row[0];
    } else {
      Bm(nm + 1, 1) = 1.0;
      Bm(1, nm + 1) = 1.0;
      for (int i = 1; i <= nm - 1; ++i) {
        Bm(nm + 1, i + 1) = row[i - 1];
        Bm(i + 1, nm + 1) = row[i - 1];
      }
      Bm(nm + 1, nm + 1) = row[nm - 1];
    }
    const int n1 = nm + 1;
    for (int kk = 1; kk <= n1; ++kk)
      for (int j = 1; j <= n1; ++j) ga[(kk - 1) * n1 + (j - 1)] = Bm(j, kk);
    for (int j = 0; j < n1; ++j) gb[j] = 0.0;
    gb[0] = 1.0;
  }
  __syncwarp();
  const bool ok = gjinv_warp(nm + 1, ga, gb, gpiv);
  if (threadIdx.x == 0) {
    int* sl = bs.slot + (size_t)k * nd;
    if (nm_old >= nd)
      for (int j = 0; j < nd; ++j) sl[j] = pm[j];
    double* cf = bs.coef + (size_t)k * kMaxHist;
    if (ok) {
      for (int h = 0; h < nm; ++h) cf[h] = gb[h + 1];
      bs.nmat[k] = nm + 1;
    } else {  // singular: restart the history (jacobi_diis.f90:214-217)
      bs.nmat[k] = 1;
      bs.restarts[k] += 1;
    }
    bs.ext[k] = ok ? nm : -nm;
  }
}

// DIIS extrapolation (jacobi_diis.f90:222-226) or, after a singular Gram
// system, the Jacobi iterate; increment H-norm (hnorm) and update.
template <class H>
__global__ void __launch_bounds__(kSolT) k_batch_extrap(const YlmTables tb, BatchState bs,
                                                        double* x) {
  const int c = blockIdx.x, k = bs.cmol[c];
  if (bs.status[k] != 0) return;
  __shared__ int pm[kMaxHist];
  __shared__ double cf[kMaxHist];
  __shared__ double tot[1];
  const int ext = bs.ext[k], nm = ext > 0 ? ext : -ext;
  const bool ok = ext > 0;
  if (threadIdx.x < nm) {
    pm[threadIdx.x] = bs.slot[(size_t)k * bs.ndiis + threadIdx.x];
    cf[threadIdx.x] = ok ? bs.coef[(size_t)k * kMaxHist + threadIdx.x] : 0.0;
  }
  __syncthreads();
  const int nylm = tb.nylm;
  const long long N = bs.n_total;
  const long long b0 = (long long)bs.off[k] * nylm + (long long)(c - bs.cfirst[k]) * kBChunk;
  const int cnt = (int)min((long long)kBChunk, (long long)bs.off[k + 1] * nylm - b0);
  const H* xjac = static_cast<const H*>(bs.hx) + (size_t)pm[nm - 1] * N + b0;
  const int dt = kSolT % nylm;
  double acc = 0.0;
#pragma unroll
  for (int u0 = 0; u0 < kBChunk / kSolT; u0 += kSolU) {
    double xo[kSolU];
    bool in[kSolU];
#pragma unroll
    for (int u = 0; u < kSolU; ++u) {
      in[u] = threadIdx.x + (u0 + u) * kSolT < cnt;
      xo[u] = 0.0;
    }
    if (ok) {
#pragma unroll 4
      for (int h = 0; h < nm; ++h) {
        const H* hk = static_cast<const H*>(bs.hx) + (size_t)pm[h] * N + b0;
        H hv[kSolU];
#pragma unroll
        for (int u = 0; u < kSolU; ++u)
          hv[u] = in[u] ? hk[threadIdx.x + (u0 + u) * kSolT] : H(0);
#pragma unroll
        for (int u = 0; u < kSolU; ++u) xo[u] = fma(cf[h], (double)hv[u], xo[u]);
      }
    } else {
#pragma unroll
      for (int u = 0; u < kSolU; ++u)
        xo[u] = in[u] ? (double)xjac[threadIdx.x + (u0 + u) * kSolT] : 0.0;
    }
    int lm = (int)((b0 + threadIdx.x + u0 * kSolT) % nylm);
#pragma unroll
    for (int u = 0; u < kSolU; ++u) {
      if (in[u]) {
        const long long q = b0 + threadIdx.x + (u0 + u) * kSolT;
        const double dd = xo[u] - x[q];
        acc = fma(dd * dd, 1.0 / (1.0 + l_of(lm)), acc);
        x[q] = xo[u];
      }
      lm = lm_add(lm, dt, nylm);
    }
  }
  double v[1] = {acc};
  block_sum_store<1, kMaxHist + 1>(v, 1, bs.part);  // chunk c is block c
  if (!batch_last_chunk(bs, k)) return;
  batch_sum_parts(bs, k, 1, tot);
  if (threadIdx.x == 0) {
    const int nsph = bs.off[k + 1] - bs.off[k];
    const double nrm = sqrt(tot[0] / (double)max(nsph, 1));
    bs.norm[k] = nrm;
    const int it = bs.iters[k] + 1;
    bs.iters[k] = it;
    const double tol = bs.tolk ? bs.tolk[k] : bs.tol;
    const int mx = bs.maxk ? bs.maxk[k] : bs.max_iter;
    bs.status[k] = (nrm < tol) ? 1 : (it >= mx ? 2 : (isfinite(nrm) ? 0 : 3));
  }
}
cudaError_t launch_batch_diis(Launch L, const YlmTables& tb, const BatchState& bs,
                              const double* rhs, const double* y, double* x) {
  if (bs.nchunk == 0) return cudaSuccess;
  if (bs.f32) {
    k_batch_gram<float><<<bs.nchunk, kSolT, 0, L.st>>>(tb, bs, rhs, y, x);
    k_batch_extrap<float><<<bs.nchunk, kSolT, 0, L.st>>>(tb, bs, x);
  } else {
    k_batch_gram<double><<<bs.nchunk, kSolT, 0, L.st>>>(tb, bs, rhs, y, x);
    k_batch_extrap<double><<<bs.nchunk, kSolT, 0, L.st>>>(tb, bs, x);
  }
  *L.launches += 2;
  return cudaGetLastError();
}

__global__ void __launch_bounds__(kSolT) k_batch_residual(const YlmTables tb, BatchState bs,
                                                          const int* __restrict__ run,
                                                          const double* __restrict__ rhs,
                                                          const double* __restrict__ y,
                                                          const double* __restrict__ x,
                                                          double* r, double* d, double* e,
                                                          double* norm) {
  const int c = blockIdx.x, k = bs.cmol[c];
  if (run[k] != 0) return;
  __shared__ double tot[1];
  const int nylm = tb.nylm, dt = kSolT % nylm;
  const long long b0 = (long long)bs.off[k] * nylm + (long long)(c - bs.cfirst[k]) * kBChunk;
  const int cnt = (int)min((long long)kBChunk, (long long)bs.off[k + 1] * nylm - b0);
  int lm = (int)((b0 + threadIdx.x) % nylm);
  double acc = 0.0;
#pragma unroll 2
  for (int j = threadIdx.x; j < kBChunk; j += kSolT) {
    if (j < cnt) {
      const long long q = b0 + j;
      const int l = l_of(lm);
      const double rr = rhs[q] - y[q] - x[q] / tb.facl[l];
      const double dd = tb.facl[l] * rr;
      r[q] = rr;
      d[q] = dd;
      e[q] = dd;
      acc = fma(dd * dd, 1.0 / (1.0 + l), acc);
    }
    lm = lm_add(lm, dt, nylm);
  }
  double v[1] = {acc};
  block_sum_store<1, kMaxHist + 1>(v, 1, bs.part);
  if (!batch_last_chunk(bs, k)) return;
  batch_sum_parts(bs, k, 1, tot);
  if (threadIdx.x == 0) {
    const int nsph = bs.off[k + 1] - bs.off[k];
    norm[k] = sqrt(tot[0] / (double)max(nsph, 1));
  }
}
cudaError_t launch_batch_residual(Launch L, const YlmTables& tb, const BatchState& bs,
                                  const int* run, const double* rhs, const double* y,
                                  const double* x, double* r, double* d, double* e,
                                  double* norm) {
  if (bs.nchunk == 0) return cudaSuccess;
  k_batch_residual<<<bs.nchunk, kSolT, 0, L.st>>>(tb, bs, run, rhs, y, x, r, d, e, norm);
  ++*L.launches;
  return cudaGetLastError();
}

__global__ void __launch_bounds__(kSolT) k_batch_update(const BatchState bs, int nylm,
                                                        const int* __restrict__ upd,
                                                        const double* __restrict__ e, double* x) {
  const int c = blockIdx.x, k = bs.cmol[c];
  if (upd[k] == 0) return;
  const long long b0 = (long long)bs.off[k] * nylm + (long long)(c - bs.cfirst[k]) * kBChunk;
  const int cnt = (int)min((long long)kBChunk, (long long)bs.off[k + 1] * nylm - b0);
  for (int j = threadIdx.x; j < cnt; j += kSolT) x[b0 + j] += e[b0 + j];
}
cudaError_t launch_batch_update(Launch L, const BatchState& bs, int nylm, const int* upd,
                                const double* e, double* x) {
  if (bs.nchunk == 0) return cudaSuccess;
  k_batch_update<<<bs.nchunk, kSolT, 0, L.st>>>(bs, nylm, upd, e, x);
  ++*L.launches;
  return cudaGetLastError();
}

// per-molecule <a, b> (energy: fep * <X, psi>, cosmo.f90:155)
__global__ void k_batch_dot(const int* __restrict__ off, int nylm, const double* __restrict__ a,
                            const double* __restrict__ b, double scale, double* out) {
  const int k = blockIdx.x;
  const long long e0 = (long long)off[k] * nylm, e1 = (long long)off[k + 1] * nylm;
  double acc = 0.0;
  for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) acc = fma(a[e], b[e], acc);
  __shared__ double sh[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) sh[w] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) t += sh[ww];
    out[k] = scale * t;
  }
}
cudaError_t launch_batch_dot(Launch L, int nmol, const int* off, int nylm, const double* a,
                             const double* b, double scale, double* out) {
  if (nmol == 0) return cudaSuccess;
  k_batch_dot<<<nmol, 256, 0, L.st>>>(off, nylm, a, b, scale, out);
  ++*L.launches;
  return cudaGetLastError();
}

// source ranges of the batched N-body sums: a cavity point sums over the
// nuclei of its molecule, a nucleus over the cavity points of its molecule
__global__ void k_batch_ranges(int nsph, int ngrid, int ncav, const int2* __restrict__ mrange,
                               const int* __restrict__ cavpt, const int* __restrict__ cavoff,
                               int2* tr_cav, int2* tr_nuc) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < ncav) tr_cav[e] = mrange[cavpt[e] / ngrid];
  if (e < nsph) {
    int2 r = mrange[e];
    tr_nuc[e] = make_int2(cavoff[r.x], cavoff[r.y]);
  }
}
cudaError_t launch_batch_ranges(Launch L, int nsph, int ngrid, int ncav, const int2* mrange,
                                const int* cavpt, const int* cavoff, int2* tr_cav,
                                int2* tr_nuc) {
  long long n = max((long long)ncav, (long long)nsph);
  if (n == 0) return cudaSuccess;
  k_batch_ranges<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(nsph, ngrid, ncav, mrange, cavpt,
                                                                 cavoff, tr_cav, tr_nuc);
  ++*L.launches;
  return cudaGetLastError();
}

// FP64 peak probe: 8 independent FMA chains per thread, register resident.
template <class T>
__global__ void __launch_bounds__(256) k_fma_probe(int iters, T* out) {
  T a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = T(1) + T(1e-6) * T(threadIdx.x + k);
  const T b = T(0.999999), c = T(1e-7);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == T(12345)) out[0] = s;  // keeps the chains live
}
cudaError_t launch_fp64_probe(Launch L, int blocks, int iters, double* out) {
  k_fma_probe<double><<<blocks, 256, 0, L.st>>>(iters, out);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_fp32_probe(Launch L, int blocks, int iters, float* out) {
  k_fma_probe<float><<<blocks, 256, 0, L.st>>>(iters, out);
  ++*L.launches;
  return cudaGetLastError();
}

}  // namespace ddc

namespace ddc {
// ---------------------------------------------------------------------------
// Solute potential and field at the cavity points with a near / far split
// (mkrhs.f90:102-114 and the field of efld.f90:97-114 at the cavity,
// main.f90:241).  Every cavity point lies on its sphere's surface,
// p = c_i + r_i s_n.  A charge q_j farther than rho * r_i from c_i contributes,
// by the addition theorem (|p - c_j| > r_i = |p - c_i|),
//   q_j / |p - c_j| = sum_lm [q_j / d (4 pi / (2l+1)) t^l Y_lm(d^)] Y_lm(s_n),
//   t = r_i / d <= 1 / rho,  d = c_j - c_i,
// so the far charges of sphere i are summed once into its local expansion
//   A_lm(i) = sum_{far j} q_j / d (4 pi / (2l+1)) t^l Y_lm(d^)   (degree P)
// and evaluated at its cavity points: phi_far = sum_lm A_lm Y_lm(s_n) and
// E_far = -(1 / r_i) sum_lm A_lm grad R_lm(s_n), with R_lm(u) = |u|^l Y_lm(u^)
// the regular solid harmonic.  The accumulation of A is the L* machinery
// (the adjrhs sum "weight * 4 pi/(2l+1) t^l Y_lm(s)" over (point, source)
// pairs) with the weight -q_j / d.  The near charges (and the sphere's own)
// are summed directly.  Truncation: at most t^(P+1) / (1 - t) of each far
// term, 1e-10 for P = 10, rho = 8.
// ---------------------------------------------------------------------------
// The L* half of the normalised recurrence of the fused pass, FP64:
// Q_l = ct Q_{l-1} - Bn t^2 Q_{l-2} (three operations per value; the scale
// gam_lm sits in Kg, applied when the rows are stored), accumulated into the
// column's register rows (layout of ls_column)
template <int LMAX, int M, int OFF>
__device__ __forceinline__ void fa_column(const YlmTables& tb, double ct, double t2, double q0,
                                          double cm, double sm, double* acc) {
  constexpr int NM = LMAX + 1 - M;
  double q1 = 0.0;
#pragma unroll
  for (int l = M; l <= LMAX; ++l) {
    double Q;
    if (l == M) {
      Q = q0;
    } else if (l == M + 1) {
      q1 = ct * q0;
      Q = q1;
    } else {
      Q = fma(ct, q1, -(tb.Bn[lmi(l, M)] * t2) * q0);
      q0 = q1;
      q1 = Q;
    }
    if (M == 0) {
      acc[OFF + l] += Q;
    } else {
      acc[OFF + (l - M)] = fma(Q, cm, acc[OFF + (l - M)]);
      acc[OFF + NM + (l - M)] = fma(Q, sm, acc[OFF + NM + (l - M)]);
    }
  }
}
// Roles of k_far_acc: at lmax 10 four roles of about three columns each
// (the greedy map of the FP32 fused pass: each role's per-source fixed cost
// paid four times instead of six), else the pairing m / lmax-m
__host__ __device__ constexpr bool fa_greedy(int L) { return L == 10; }
__host__ __device__ constexpr int fa_nroles(int L) { return fa_greedy(L) ? 4 : L / 2 + 1; }
template <int LMAX, int R, int M>
__device__ __forceinline__ void fa_cols(const YlmTables& tb, const double* sh, int stride, int q,
                                        double ct, double t2, double* acc) {
  constexpr int NR = fa_nroles(LMAX);
  constexpr bool G = fa_greedy(LMAX);
  if constexpr (lxs_role_of(LMAX, NR, M, G) == R)
    fa_column<LMAX, M, lxs_off_of(LMAX, NR, M, G)>(tb, ct, t2, sh[(2 + 3 * M) * stride + q],
                                                   sh[(3 + 3 * M) * stride + q],
                                                   sh[(4 + 3 * M) * stride + q], acc);
  if constexpr (M < LMAX) fa_cols<LMAX, R, M + 1>(tb, sh, stride, q, ct, t2, acc);
}
template <int LMAX, int R>
__device__ __forceinline__ void fa_role(const YlmTables& tb, const double* sh, int stride,
                                        int count, int lane, double* acc) {
  for (int q = lane; q < count; q += 32) {
    const double ct = sh[q], t2 = sh[stride + q];
    fa_cols<LMAX, R, 0>(tb, sh, stride, q, ct, t2, acc);
  }
}
template <int LMAX, int R>
__device__ __forceinline__ void fa_run_role(int role, const YlmTables& tb, const double* sh,
                                            int stride, int count, int lane, double* acc) {
  if (role == R) {
    fa_role<LMAX, R>(tb, sh, stride, count, lane, acc);
    return;
  }
  if constexpr (R + 1 < fa_nroles(LMAX))
    fa_run_role<LMAX, R + 1>(role, tb, sh, stride, count, lane, acc);
}

// A(i, lm) for every sphere with cavity points: block per sphere, role warps
// over chunks of the sources of its molecule.  Per source the thread forms
// 1/d and 1/sin(theta) with the refined hardware reciprocal square root
// (rsqrt_pos), the prefix and cos/sin(m phi) (the fields of k_lstarx); the
// roles run the normalised recurrence (fa_column) and store with Kg.
template <int LMAX>
__global__ void __launch_bounds__(32 * fa_nroles(LMAX), fa_greedy(LMAX) ? 4 : 1)
    k_far_acc(const YlmTables tb, int nsph,
                                                                   const double4* __restrict__ sph,
                                                                   const double* __restrict__ q,
                                                                   const int2* __restrict__ mrange,
                                                                   const int* __restrict__ cavoff,
                                                                   double rho, double* A) {
  constexpr int NR = fa_nroles(LMAX);
  constexpr int CH = 32 * NR;
  constexpr int NVM = lxs_max_nvals(LMAX, NR, fa_greedy(LMAX));
  extern __shared__ double sh[];  // [ls_nfields][CH]
  const int i = blockIdx.x;
  if (cavoff[i + 1] == cavoff[i]) return;  // buried: A(i) is never read
  const int role = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double4 ci = sph[i];
  const double cut2 = (rho * ci.w) * (rho * ci.w);
  const int lo = mrange ? mrange[i].x : 0, hi = mrange ? mrange[i].y : nsph;
  double acc[NVM];
#pragma unroll
  for (int v = 0; v < NVM; ++v) acc[v] = 0.0;
  for (int j0 = lo; j0 < hi; j0 += CH) {
    const int chunk = min(CH, hi - j0);
    {
      const int tt = threadIdx.x;
      double* col = sh + tt;
      double ct = 0.0, t2 = 0.0, st = 0.0, w = 0.0, cp = 1.0, sp = 0.0;
      if (tt < chunk) {
        const int j = j0 + tt;
        const double4 cj = sph[j];
        const double vx = cj.x - ci.x, vy = cj.y - ci.y, vz = cj.z - ci.z;
        const double d2 = vx * vx + vy * vy + vz * vz;
        if (j != i && d2 > cut2) {
          const double di = rsqrt_pos(d2);
          const double t = ci.w * di, c = vz * di;
          const double s2 = fma(-c, c, 1.0);
          double sn = 0.0;
          if (s2 > 1e-280) {  // off the pole (at a pole only m = 0 survives)
            const double rs = rsqrt_pos(s2);
            sn = s2 * rs;
            cp = vx * di * rs;
            sp = vy * di * rs;
          }
          ct = c * t;
          t2 = t * t;
          st = sn * t;
          w = -q[j] * di;
        }
      }
      col[0] = ct;
      col[CH] = t2;
      double pmm = w, cm = 1.0, sm = 0.0, cmm1 = 1.0, smm1 = 0.0;
#pragma unroll
      for (int m = 0; m <= LMAX; ++m) {
        if (m == 1) {
          cm = cp;
          sm = sp;
        } else if (m >= 2) {
          const double cn = 2.0 * cp * cm - cmm1, sn = 2.0 * cp * sm - smm1;
          cmm1 = cm; smm1 = sm; cm = cn; sm = sn;
        }
        col[(2 + 3 * m) * CH] = pmm;
        col[(3 + 3 * m) * CH] = cm;
        col[(4 + 3 * m) * CH] = sm;
        pmm = -pmm * (2.0 * m + 1.0) * st;
      }
    }
    __syncthreads();
    fa_run_role<LMAX, 0>(role, tb, sh, CH, chunk, lane, acc);
    __syncthreads();
  }
  lxs_finish_role<LMAX, NR, 0, double, true, fa_greedy(LMAX)>(role, tb, acc,
                                                              A + (size_t)i * tb.nylm, lane);
}

// Tables on the grid, once per context: BT[lm][n] = Y_lm(s_n) and
// DT[k][lm][n] = d R_lm / d u_k at u = s_n (k = x, y, z), by fourth-order
// central differences of R_lm(u) = |u|^l Y_lm(u / |u|) with step 1e-4
// (truncation ~h^4 l^5 / 30 and rounding ~1e-16 / h: about 1e-12 relative)
__global__ void k_far_tables(const YlmTables tb, const double4* __restrict__ grid, int ngrid,
                             double* BT, double* DT) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 4 * ngrid) return;
  const int n = e % ngrid, k = e / ngrid;  // k = 0: values; 1..3: d/du_{k-1}
  const double4 g = grid[n];
  const int ny = tb.nylm;
  double y[(DDC_MAX_LMAX + 1) * (DDC_MAX_LMAX + 1)];
  if (k == 0) {
    ylmbas_ref(tb, g.x, g.y, g.z, y);
    for (int lm = 0; lm < ny; ++lm) BT[(size_t)lm * ngrid + n] = y[lm];
    return;
  }
  double acc[(DDC_MAX_LMAX + 1) * (DDC_MAX_LMAX + 1)];
  for (int lm = 0; lm < ny; ++lm) acc[lm] = 0.0;
  const double h = 1e-4;
  const double cst[4] = {1.0, -8.0, 8.0, -1.0};   // f(-2h), f(-h), f(h), f(2h)
  const double off[4] = {-2.0, -1.0, 1.0, 2.0};
  for (int s = 0; s < 4; ++s) {
    double u[3] = {g.x, g.y, g.z};
    u[k - 1] += off[s] * h;
    const double r = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    ylmbas_ref(tb, u[0] / r, u[1] / r, u[2] / r, y);
    double rl = 1.0;
    for (int l = 0; l <= tb.lmax; ++l) {
      for (int m = -l; m <= l; ++m) acc[l * l + l + m] += cst[s] * rl * y[l * l + l + m];
      rl *= r;
    }
  }
  for (int lm = 0; lm < ny; ++lm)
    DT[((size_t)(k - 1) * ny + lm) * ngrid + n] = acc[lm] / (12.0 * h);
}

// Potential and field at the cavity points of sphere i (block per sphere):
// the near charges directly (compacted into shared memory in passes of at
// most kNearCap), the far ones from A(i).  With ef == nullptr only phi.  A
// sphere without cavity points (buried) has nothing to do; the others run
// with NU = ceil(points / 128) point slots per thread (a sphere has 90
// points on average at the 20k workload, up to 590), so no thread steps
// through empty slots in the pair loop.
constexpr int kNearCap = 1024;
constexpr int kCandGroups = 512;
template <int NU>
__device__ __forceinline__ void far_cav_body(int i, int ngrid, int ny, double4 ci, double cut2,
                                             int lo, int hi, int c0, int c1,
                                             const double4* __restrict__ sph,
                                             const double* __restrict__ q,
                                             const int* __restrict__ cavpt,
                                             const double* __restrict__ ccav,
                                             const double* __restrict__ BT,
                                             const double* __restrict__ DT, double* phi,
                                             double* ef, double4* near, const double* sA,
                                             int& s_cnt, int& s_scan, int* wbase,
                                             const int* cgl, const int* cpre, int ncg,
                                             const int* __restrict__ gsph,
                                             const int* __restrict__ gstart) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  // candidate f of the scan: sphere f of the molecule's range, or with cell
  // groups (ncg > 0) the member f - cpre[k] of candidate group cgl[k]
  auto cand = [&](int f) -> int {
    if (ncg == 0) return f;
    int a = 0, b = ncg;  // cpre[a] <= f < cpre[b]
    while (b - a > 1) {
      const int mid = (a + b) >> 1;
      if (cpre[mid] <= f) a = mid;
      else b = mid;
    }
    return gsph[gstart[cgl[a]] + (f - cpre[a])];
  };
  // thread tid owns cavity points c0 + tid + 128 u, u < NU
  double v[NU], ex[NU], ey[NU], ez[NU], px[NU], py[NU], pz[NU];
#pragma unroll
  for (int u = 0; u < NU; ++u) {
    v[u] = ex[u] = ey[u] = ez[u] = 0.0;
    const int c = c0 + tid + 128 * u;
    px[u] = py[u] = pz[u] = 0.0;
    if (c < c1) {
      px[u] = ccav[3 * (size_t)c];
      py[u] = ccav[3 * (size_t)c + 1];
      pz[u] = ccav[3 * (size_t)c + 2];
    }
  }
  if (tid == 0) s_scan = lo;
  __syncthreads();
  // passes over the molecule: compact near charges, then sum them
  while (true) {
    if (tid == 0) s_cnt = 0;
    __syncthreads();
    const int start = s_scan;
    if (start >= hi) break;
    int j = start;
    // scan in steps of 128 candidates while the buffer has room for a step
    for (; j < hi; j += 128) {
      __syncthreads();
      if (s_cnt + 128 > kNearCap) break;
      const int jj = j + tid;
      bool nb = false;
      double4 cj = make_double4(0, 0, 0, 0);
      int js = 0;
      if (jj < hi) {
        js = cand(jj);
        cj = sph[js];
        const double dx = cj.x - ci.x, dy = cj.y - ci.y, dz = cj.z - ci.z;
        nb = js == i || dx * dx + dy * dy + dz * dz <= cut2;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, nb);
      if (lane == 0) wbase[w] = __popc(bal);
      __syncthreads();
      if (tid == 0) {
        int b = s_cnt;
        for (int k = 0; k < 4; ++k) {
          const int c = wbase[k];
          wbase[k] = b;
          b += c;
        }
        s_cnt = b;
      }
      __syncthreads();
      if (nb) near[wbase[w] + __popc(bal & ((1u << lane) - 1u))] = make_double4(cj.x, cj.y, cj.z, q[js]);
    }
    __syncthreads();
    if (tid == 0) s_scan = j;
    const int cnt = s_cnt;
    for (int k = 0; k < cnt; ++k) {
      const double4 s = near[k];
#pragma unroll
      for (int u = 0; u < NU; ++u) {
        if (c0 + tid + 128 * u < c1) {
          const double dx = px[u] - s.x, dy = py[u] - s.y, dz = pz[u] - s.z;
          const double ri = rsqrt_pos(dx * dx + dy * dy + dz * dz);
          v[u] = fma(s.w, ri, v[u]);
          const double f = s.w * (ri * ri * ri);
          ex[u] = fma(f, dx, ex[u]);
          ey[u] = fma(f, dy, ey[u]);
          ez[u] = fma(f, dz, ez[u]);
        }
      }
    }
    __syncthreads();
  }
  // far part from the local expansion
  const double iri = 1.0 / ci.w;
#pragma unroll
  for (int u = 0; u < NU; ++u) {
    const int c = c0 + tid + 128 * u;
    if (c >= c1) continue;
    const int n = cavpt[c] - i * ngrid;
    double fp = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
    for (int lm = 0; lm < ny; ++lm) {
      const double a = sA[lm];
      fp = fma(a, BT[(size_t)lm * ngrid + n], fp);
      if (ef) {
        fx = fma(a, DT[(size_t)lm * ngrid + n], fx);
        fy = fma(a, DT[((size_t)ny + lm) * ngrid + n], fy);
        fz = fma(a, DT[((size_t)2 * ny + lm) * ngrid + n], fz);
      }
    }
    phi[c] = v[u] + fp;
    if (ef) {
      ef[3 * (size_t)c] = ex[u] - iri * fx;
      ef[3 * (size_t)c + 1] = ey[u] - iri * fy;
      ef[3 * (size_t)c + 2] = ez[u] - iri * fz;
    }
  }
}

__global__ void __launch_bounds__(128) k_far_cav(int nsph, int ngrid, int ny,
                                                 const double4* __restrict__ sph,
                                                 const double* __restrict__ q,
                                                 const int2* __restrict__ mrange, double rho,
                                                 const int* __restrict__ cavoff,
                                                 const int* __restrict__ cavpt,
                                                 const double* __restrict__ ccav,
                                                 const double* __restrict__ A,
                                                 const double* __restrict__ BT,
                                                 const double* __restrict__ DT, double* phi,
                                                 double* ef, const ZGroups zg) {
  __shared__ double4 near[kNearCap];
  __shared__ double sA[(DDC_MAX_LMAX + 1) * (DDC_MAX_LMAX + 1)];
  __shared__ int s_cnt, s_scan, wbase[4];
  __shared__ int cgl[kCandGroups], cpre[kCandGroups + 1];
  __shared__ int s_ncg;
  const int i = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int c0 = cavoff[i], c1 = cavoff[i + 1];
  if (c1 == c0) return;  // buried: no cavity points
  const double4 ci = sph[i];
  const double cut2 = (rho * ci.w) * (rho * ci.w);
  int lo = mrange ? mrange[i].x : 0, hi = mrange ? mrange[i].y : nsph;
  for (int lm = tid; lm < ny; lm += blockDim.x) sA[lm] = A[(size_t)i * ny + lm];
  // with cell groups (one molecule): the groups that can hold a near charge
  // (|c_i - c_g| <= rho r_i + R_g, R_g bounding the members' centres; 1e-6
  // bohr of margin for rounding), compacted in group order, and the prefix
  // sums of their sizes; more than kCandGroups keeps the full scan
  int ncg = 0;
  if (zg.ngroup > 0) {
    if (tid == 0) s_ncg = 0;
    __syncthreads();
    const double reach = rho * ci.w;
    for (int g0 = 0; g0 < zg.ngroup; g0 += 128) {
      const int g = g0 + tid;
      bool c = false;
      if (g < zg.ngroup) {
        const double4 cg = zg.gcen[g];
        const double dx = ci.x - cg.x, dy = ci.y - cg.y, dz = ci.z - cg.z;
        const double lim = reach + cg.w + 1e-6;
        c = dx * dx + dy * dy + dz * dz <= lim * lim;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, c);
      if (lane == 0) wbase[w] = __popc(bal);
      __syncthreads();
      if (tid == 0) {
        int b = s_ncg;
        for (int k = 0; k < 4; ++k) {
          const int n = wbase[k];
          wbase[k] = b;
          b += n;
        }
        s_ncg = b;
      }
      __syncthreads();
      const int pos = wbase[w] + __popc(bal & ((1u << lane) - 1u));
      if (c && pos < kCandGroups) cgl[pos] = g;
      __syncthreads();
    }
    ncg = s_ncg;
    if (ncg <= kCandGroups) {
      // prefix sums of the candidate groups' sizes (warp 0, in order)
      if (w == 0) {
        int run = 0;
        for (int k0 = 0; k0 < ncg; k0 += 32) {
          const int k = k0 + lane;
          int v = k < ncg ? zg.gstart[cgl[k] + 1] - zg.gstart[cgl[k]] : 0;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
          }
          if (k < ncg) cpre[k + 1] = run + v;
          run += __shfl_sync(0xffffffffu, v, 31);
        }
        if (lane == 0) cpre[0] = 0;
      }
      __syncthreads();
      lo = 0;
      hi = ncg > 0 ? cpre[ncg] : 0;
    } else {
      ncg = 0;  // too many candidates: scan the molecule
    }
  }
  // 5 * 128 = 640 >= ngrid up to 590 points
  switch ((c1 - c0 + 127) / 128) {
#define FAR_CAV_CASE(NU)                                                                        \
  case NU:                                                                                      \
    far_cav_body<NU>(i, ngrid, ny, ci, cut2, lo, hi, c0, c1, sph, q, cavpt, ccav, BT, DT, phi, \
                     ef, near, sA, s_cnt, s_scan, wbase, cgl, cpre, ncg, zg.gsph, zg.gstart);  \
    break;
    FAR_CAV_CASE(1)
    FAR_CAV_CASE(2)
    FAR_CAV_CASE(3)
    FAR_CAV_CASE(4)
    FAR_CAV_CASE(5)
#undef FAR_CAV_CASE
    default:
      break;
  }
}

cudaError_t launch_far_tables(Launch L, const YlmTables& tbP, const double4* grid, int ngrid,
                              double* BT, double* DT) {
  const int n = 4 * ngrid;
  k_far_tables<<<(n + 63) / 64, 64, 0, L.st>>>(tbP, grid, ngrid, BT, DT);
  ++*L.launches;
  return cudaGetLastError();
}

cudaError_t launch_far_pot_field(Launch L, const YlmTables& tbP, int nsph, int ngrid,
                                 const double4* sph, const double* q, const int2* mrange,
                                 double rho, const int* cavoff, const int* cavpt,
                                 const double* ccav, const double* BT, const double* DT,
                                 double* A, double* phi, double* ef, const ZGroups* zg) {
  if (nsph == 0) return cudaSuccess;
  if (ngrid > 640) return cudaErrorInvalidValue;  // k_far_cav holds 5 x 128 points per thread set
  cudaError_t e;
#define CASE(LV)                                                                              \
  case LV: {                                                                                  \
    constexpr int NR = fa_nroles(LV);                                                         \
    const size_t sm = sizeof(double) * ls_nfields(LV) * 32 * NR;                              \
    if (sm > 48 * 1024)                                                                       \
      if ((e = cudaFuncSetAttribute(k_far_acc<LV>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                    (int)sm)))                                                \
        return e;                                                                             \
    k_far_acc<LV><<<nsph, 32 * NR, sm, L.st>>>(tbP, nsph, sph, q, mrange, cavoff, rho, A);    \
    break;                                                                                    \
  }
  switch (tbP.lmax) {
    DDC_LMAX_CASES(CASE)
    default:
      return cudaErrorInvalidValue;
  }
#undef CASE
  ++*L.launches;
  if ((e = cudaGetLastError())) return e;
  ZGroups none;
  k_far_cav<<<nsph, 128, 0, L.st>>>(nsph, ngrid, tbP.nylm, sph, q, mrange, rho, cavoff, cavpt,
                                    ccav, A, BT, DT, phi, ef, zg && !mrange ? *zg : none);
  ++*L.launches;
  return cudaGetLastError();
}

}  // namespace ddc
