// ddc_zfar.cu -- the field of the cavity charges zeta at the nuclei
// (efld.f90:97-114 as called at main.f90:259-265) with a grouped multipole
// far field, for large molecules in the mixed-precision flow.
//
// This field enters only the forces, and the mixed flow already sums it
// with FP32 pair arithmetic (k_efield_f2).  Direct, it costs N * ncav pairs
// (3.6e10 at 20,000 spheres).  Here the spheres are grouped by the cells of
// a uniform grid over their centres (Morton order of the cells, at most 16
// per dimension, side >= kZetaCell), and each group's cavity charges get a
// multipole expansion of degree P = kZetaDegree about the group's centroid:
//   M_n^m = sum_k zeta_k conj(R_n^m((p_k - c_g) / a)),   a = group radius,
//   R_n^m(v) = |v|^n P_n^m(cos theta) e^{i m phi} / (n+m)!   (regular),
//   I_n^m(v) = (n-m)! P_n^m(cos theta) e^{i m phi} / |v|^{n+1} (irregular),
// P_n^m without the Condon-Shortley phase, I_n^{-m} = conj(I_n^m).  With
// these scalings 1 / |x - p| = sum_{n,m} conj(R_n^m(p)) I_n^m(x) for |p| <
// |x| (the Legendre addition theorem), and the derivatives close on the
// irregular harmonics:  d/dz I_n^m = -I_{n+1}^m,  (d/dx + i d/dy) I_n^m =
// -I_{n+1}^{m+1},  (d/dx - i d/dy) I_n^m = I_{n+1}^{m-1} (m >= 1).  So the
// field E = -grad Phi of a group at v = (x - c_g) / a is, times 1 / a^2,
//   E_z        = sum_n [M_n^0 I_{n+1}^0 + 2 Re sum_{m>=1} M_n^m I_{n+1}^m],
//   E_x + iE_y = sum_n [sum_{m>=0} M_n^m I_{n+1}^{m+1}
//                       - sum_{m>=1} conj(M_n^m I_{n+1}^{m-1})].
// A nucleus farther than kZetaRho * a from a group's centroid takes the
// group's expansion (truncation below (1/3)^17 / (1 - 1/3) = 1.2e-8 of the
// group's charge scale, under the FP32 rounding of the pair sums); a warp
// whose 32 nuclei are not all far sums the group's points directly (FP32
// pairs as in k_efield_f2, in warp tiles of 32 points staged in shared
// memory, flushed to FP64 every 256 points).  The moments
// are accumulated in FP64 and stored in FP32 (scaled coordinates keep every
// term of order one); the evaluation runs in FP32 and each group's
// contribution is added in FP64.  Every sum has a fixed order: per target,
// groups in order within a chunk of kZChunk groups, chunks reduced in order
// by k_zg_reduce.  No atomics on values: the result is bit-reproducible.
#include <cfloat>

#include "ddc_internal.h"

namespace ddc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kZP = kZetaDegree;
constexpr int kZNM = (kZP + 1) * (kZP + 2) / 2;  // n <= P, 0 <= m <= n
constexpr int kZCells = 4096;                    // 16 x 16 x 16 cells
constexpr int kZChunk = 16;                      // groups per block of the field kernel
constexpr int kZTile = 128;                      // nuclei per block
__host__ __device__ constexpr int zidx(int n, int m) { return n * (n + 1) / 2 + m; }

__device__ __forceinline__ int zg_morton(int ix, int iy, int iz) {
  int c = 0;
#pragma unroll
  for (int b = 0; b < 4; ++b)
    c |= (((ix >> b) & 1) << (3 * b)) | (((iy >> b) & 1) << (3 * b + 1)) |
         (((iz >> b) & 1) << (3 * b + 2));
  return c;
}

// Groups of one molecule: one block.  Bounding box of the centres, cell of
// each sphere, per-cell counts, their exclusive scan (group starts of the
// non-empty cells, in Morton order) and an ordered fill of the member lists
// (warp 0, 32 spheres at a time in index order: members of a group stay in
// increasing sphere index, whatever the thread timing).
__global__ void __launch_bounds__(1024) k_zg_build(int nsph, const double4* __restrict__ sph,
                                                   double hmin, int* __restrict__ cellid,
                                                   int* __restrict__ gsph,
                                                   int* __restrict__ gstart,
                                                   int* __restrict__ ngroup) {
  __shared__ int cnt[kZCells], cur[kZCells];
  __shared__ double red[2][3][32];
  __shared__ double s_lo[3], s_h;
  __shared__ int wsum[32], wne[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int j = tid; j < nsph; j += 1024) {
    const double4 c = sph[j];
    lo[0] = fmin(lo[0], c.x);
    lo[1] = fmin(lo[1], c.y);
    lo[2] = fmin(lo[2], c.z);
    hi[0] = fmax(hi[0], c.x);
    hi[1] = fmax(hi[1], c.y);
    hi[2] = fmax(hi[2], c.z);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      lo[k] = fmin(lo[k], __shfl_xor_sync(kFull, lo[k], o));
      hi[k] = fmax(hi[k], __shfl_xor_sync(kFull, hi[k], o));
    }
    if (lane == 0) {
      red[0][k][w] = lo[k];
      red[1][k][w] = hi[k];
    }
  }
  for (int c = tid; c < kZCells; c += 1024) cnt[c] = 0;
  __syncthreads();
  if (tid == 0) {
    double ext = 0.0;
    for (int k = 0; k < 3; ++k) {
      double a = DBL_MAX, b = -DBL_MAX;
      for (int q = 0; q < 32; ++q) {
        a = fmin(a, red[0][k][q]);
        b = fmax(b, red[1][k][q]);
      }
      s_lo[k] = a;
      ext = fmax(ext, b - a);
    }
    // at most 16 cells per dimension: floor(ext / h) <= 15
    s_h = fmax(hmin, ext / 15.5);
  }
  __syncthreads();
  const double h = s_h, lx = s_lo[0], ly = s_lo[1], lz = s_lo[2];
  for (int j = tid; j < nsph; j += 1024) {
    const double4 c = sph[j];
    const int ix = min(15, (int)((c.x - lx) / h)), iy = min(15, (int)((c.y - ly) / h)),
              iz = min(15, (int)((c.z - lz) / h));
    const int cid = zg_morton(ix, iy, iz);
    cellid[j] = cid;
    atomicAdd(&cnt[cid], 1);  // counts: order-free
  }
  __syncthreads();
  // exclusive scan of the counts (four cells per thread) and of the
  // non-empty flags (group index of each non-empty cell)
  int v[4], s = 0, ne = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cnt[4 * tid + k];
    s += v[k];
    ne += v[k] > 0;
  }
  int is = s, ine = ne;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int a = __shfl_up_sync(kFull, is, o), b = __shfl_up_sync(kFull, ine, o);
    if (lane >= o) {
      is += a;
      ine += b;
    }
  }
  if (lane == 31) {
    wsum[w] = is;
    wne[w] = ine;
  }
  __syncthreads();
  if (w == 0) {
    int a = wsum[lane], b = wne[lane];
    const int a0 = a, b0 = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(kFull, a, o), y = __shfl_up_sync(kFull, b, o);
      if (lane >= o) {
        a += x;
        b += y;
      }
    }
    wsum[lane] = a - a0;
    wne[lane] = b - b0;
  }
  __syncthreads();
  int base = wsum[w] + is - s, gi = wne[w] + ine - ne;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    cur[4 * tid + k] = base;
    if (v[k] > 0) gstart[gi++] = base;
    base += v[k];
  }
  if (tid == 1023) {
    *ngroup = gi;
    gstart[gi] = nsph;
  }
  __syncthreads();
  if (w == 0) {
    for (int j0 = 0; j0 < nsph; j0 += 32) {
      const int j = j0 + lane;
      const int cid = j < nsph ? cellid[j] : -1 - lane;
      const unsigned mask = __match_any_sync(kFull, cid);
      const int rank = __popc(mask & ((1u << lane) - 1u));
      if (j < nsph) gsph[cur[cid] + rank] = j;
      __syncwarp();
      if (j < nsph && rank == 0) cur[cid] += __popc(mask);
      __syncwarp();
    }
  }
}

// Centroid c_g and radius R_g = max |c_j - c_g| + r_j of each group; warp
// per group, fixed shuffle trees.  R_g bounds the group's cavity points (on
// the members' surfaces) and its members' overlaps: a sphere i overlapping
// a member j has |c_i - c_g| <= r_i + r_j + |c_j - c_g| <= r_i + R_g.
__global__ void __launch_bounds__(128) k_zg_geom(int ngroup, const int* __restrict__ gstart,
                                                 const int* __restrict__ gsph,
                                                 const double4* __restrict__ sph,
                                                 double4* __restrict__ gcen) {
  const int g = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (g >= ngroup) return;
  const int s0 = gstart[g], s1 = gstart[g + 1];
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int k = s0 + lane; k < s1; k += 32) {
    const double4 c = sph[gsph[k]];
    sx += c.x;
    sy += c.y;
    sz += c.z;
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    sx += __shfl_xor_sync(kFull, sx, o);
    sy += __shfl_xor_sync(kFull, sy, o);
    sz += __shfl_xor_sync(kFull, sz, o);
  }
  const double inv = 1.0 / (double)(s1 - s0);
  const double cx = sx * inv, cy = sy * inv, cz = sz * inv;
  double R = 0.0;
  for (int k = s0 + lane; k < s1; k += 32) {
    const double4 c = sph[gsph[k]];
    const double dx = c.x - cx, dy = c.y - cy, dz = c.z - cz;
    R = fmax(R, sqrt(dx * dx + dy * dy + dz * dz) + c.w);
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) R = fmax(R, __shfl_xor_sync(kFull, R, o));
  if (lane == 0) gcen[g] = make_double4(cx, cy, cz, R);
}

// cavity points per group (gnpt[G] = 0: the scan reads one past)
__global__ void __launch_bounds__(128) k_zg_npt(int ngroup, const int* __restrict__ gstart,
                                                const int* __restrict__ gsph,
                                                const int* __restrict__ cavoff,
                                                int* __restrict__ gnpt) {
  const int g = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (g == ngroup && lane == 0) gnpt[ngroup] = 0;
  if (g >= ngroup) return;
  int np = 0;
  for (int k = gstart[g] + lane; k < gstart[g + 1]; k += 32) {
    const int j = gsph[k];
    np += cavoff[j + 1] - cavoff[j];
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) np += __shfl_xor_sync(kFull, np, o);
  if (lane == 0) gnpt[g] = np;
}

// one column m of the moments for the points a thread owns: acc[n] +=
// zeta conj(R_n^m(v)), n = m..P, v the scaled point
template <int M>
__host__ __device__ __forceinline__ void zg_column(double x, double y, double z, double r2, double q,
                                          double2* acc) {
  // R_m^m = (x + iy)^m / (2^m m!)
  double rr = 1.0, ri = 0.0;
#pragma unroll
  for (int k = 1; k <= M; ++k) {
    const double s = 1.0 / (2.0 * k);
    const double a = (rr * x - ri * y) * s, b = (rr * y + ri * x) * s;
    rr = a;
    ri = b;
  }
  double pr = 0.0, pi = 0.0;  // R_{n-2}^m
#pragma unroll
  for (int n = M; n <= kZP; ++n) {
    double cr, ci;
    if (n == M) {
      cr = rr;
      ci = ri;
    } else if (n == M + 1) {
      cr = z * rr;
      ci = z * ri;
    } else {
      // R_n^m = ((2n-1) z R_{n-1}^m - r^2 R_{n-2}^m) / (n^2 - m^2)
      const double f = 1.0 / (double)(n * n - M * M);
      cr = ((2 * n - 1) * z * rr - r2 * pr) * f;
      ci = ((2 * n - 1) * z * ri - r2 * pi) * f;
    }
    if (n > M) {
      pr = rr;
      pi = ri;
    }
    rr = cr;
    ri = ci;
    acc[n].x += q * cr;
    acc[n].y -= q * ci;
  }
}

template <int M>
__device__ __forceinline__ void zg_moments_col(int s0, int s1, const int* __restrict__ gsph,
                                               const int* __restrict__ cavoff,
                                               const double* __restrict__ ccav,
                                               const double* __restrict__ zeta, double4 cg,
                                               double ia, double2 (*part)[128], float2* Mg) {
  double2 acc[kZP + 1];
#pragma unroll
  for (int n = 0; n <= kZP; ++n) acc[n] = make_double2(0.0, 0.0);
  for (int k = s0; k < s1; ++k) {
    const int j = gsph[k], c0 = cavoff[j], c1 = cavoff[j + 1];
    for (int c = c0 + (int)threadIdx.x; c < c1; c += 128) {
      const double x = (ccav[3 * (size_t)c] - cg.x) * ia, y = (ccav[3 * (size_t)c + 1] - cg.y) * ia,
                   z = (ccav[3 * (size_t)c + 2] - cg.z) * ia;
      zg_column<M>(x, y, z, x * x + y * y + z * z, zeta[c], acc);
    }
  }
#pragma unroll
  for (int n = M; n <= kZP; ++n) part[n][threadIdx.x] = acc[n];
  __syncthreads();
  const int n = M + (int)threadIdx.x;
  if (n <= kZP) {
    double2 s = make_double2(0.0, 0.0);
    for (int t = 0; t < 128; ++t) {
      s.x += part[n][t].x;
      s.y += part[n][t].y;
    }
    Mg[zidx(n, M)] = make_float2((float)s.x, (float)s.y);
  }
  __syncthreads();
  if constexpr (M < kZP)
    zg_moments_col<M + 1>(s0, s1, gsph, cavoff, ccav, zeta, cg, ia, part, Mg);
}

// Per group (block of 128): its points packed in member order as FP32
// (p - c_g, zeta), and its moments, column by column (per-thread FP64
// partials summed over the threads in thread order).
__global__ void __launch_bounds__(128) k_zg_moments(
    const int* __restrict__ gstart, const int* __restrict__ gsph, const double4* __restrict__ gcen,
    const int* __restrict__ gptr, const int* __restrict__ cavoff, const double* __restrict__ ccav,
    const double* __restrict__ zeta, float4* __restrict__ zpk, float2* __restrict__ M) {
  __shared__ double2 part[kZP + 1][128];
  const int g = blockIdx.x, tid = threadIdx.x;
  const double4 cg = gcen[g];
  const int s0 = gstart[g], s1 = gstart[g + 1];
  int off = gptr[g];
  for (int k = s0; k < s1; ++k) {
    const int j = gsph[k], c0 = cavoff[j], c1 = cavoff[j + 1];
    for (int c = c0 + tid; c < c1; c += 128)
      zpk[off + (c - c0)] = make_float4((float)(ccav[3 * (size_t)c] - cg.x),
                                        (float)(ccav[3 * (size_t)c + 1] - cg.y),
                                        (float)(ccav[3 * (size_t)c + 2] - cg.z), (float)zeta[c]);
    off += c1 - c0;
  }
  zg_moments_col<0>(s0, s1, gsph, cavoff, ccav, zeta, cg, 1.0 / cg.w, part,
                    M + (size_t)g * kZNM);
}

// contributions of I_N^k (N >= 1) to the field: moments of degree N-1
template <int N, int K>
__host__ __device__ __forceinline__ void zg_contrib(float ir, float ii, const float2* __restrict__ Mg,
                                           float& ez, float& ez2, float& epr, float& epi) {
  constexpr int n = N - 1;
  if constexpr (K <= n) {  // E_z: M_n^K I_{n+1}^K (twice for K >= 1)
    const float2 m = Mg[zidx(n, K)];
    if constexpr (K == 0) ez = fmaf(m.x, ir, fmaf(-m.y, ii, ez));
    else ez2 = fmaf(m.x, ir, fmaf(-m.y, ii, ez2));
  }
  if constexpr (K >= 1 && K - 1 <= n) {  // E_+: + M_n^{K-1} I_{n+1}^K
    const float2 m = Mg[zidx(n, K - 1)];
    epr = fmaf(m.x, ir, fmaf(-m.y, ii, epr));
    epi = fmaf(m.x, ii, fmaf(m.y, ir, epi));
  }
  if constexpr (K + 1 <= n) {  // E_+: - conj(M_n^{K+1} I_{n+1}^K)
    const float2 m = Mg[zidx(n, K + 1)];
    epr = fmaf(-m.x, ir, fmaf(m.y, ii, epr));
    epi = fmaf(m.x, ii, fmaf(m.y, ir, epi));
  }
}

// column K of the irregular harmonics, degrees K..P+1, from I_K^K
template <int K, int N>
__host__ __device__ __forceinline__ void zg_col_up(float z, float u, float i1r, float i1i, float i2r,
                                          float i2i, const float2* __restrict__ Mg, float& ez,
                                          float& ez2, float& epr, float& epi) {
  // I_N^K = u ((2N-1) z I_{N-1}^K - (N+K-1)(N-K-1) I_{N-2}^K)
  constexpr float a = (float)(2 * N - 1), b = (float)((N + K - 1) * (N - K - 1));
  const float zr = a * z;
  const float nr = u * fmaf(zr, i1r, -b * i2r), ni = u * fmaf(zr, i1i, -b * i2i);
  zg_contrib<N, K>(nr, ni, Mg, ez, ez2, epr, epi);
  if constexpr (N < kZP + 1) zg_col_up<K, N + 1>(z, u, nr, ni, i1r, i1i, Mg, ez, ez2, epr, epi);
}

template <int K>
__host__ __device__ __forceinline__ void zg_cols(float x, float y, float z, float u, float dr, float di,
                                        const float2* __restrict__ Mg, float& ez, float& ez2,
                                        float& epr, float& epi) {
  // I_K^K from I_{K-1}^K-1 (dr, di): (2K-1) (x + iy) u I_{K-1}^{K-1}
  float cr = dr, ci = di;
  if constexpr (K > 0) {
    const float s = (float)(2 * K - 1) * u;
    cr = s * (x * dr - y * di);
    ci = s * (x * di + y * dr);
    zg_contrib<K, K>(cr, ci, Mg, ez, ez2, epr, epi);
  }
  if constexpr (K + 1 <= kZP + 1) {
    // I_{K+1}^K = (2K+1) z u I_K^K
    const float s = (float)(2 * K + 1) * z * u;
    const float nr = s * cr, ni = s * ci;
    zg_contrib<K + 1, K>(nr, ni, Mg, ez, ez2, epr, epi);
    if constexpr (K + 2 <= kZP + 1)
      zg_col_up<K, K + 2>(z, u, nr, ni, cr, ci, Mg, ez, ez2, epr, epi);
  }
  if constexpr (K < kZP + 1) zg_cols<K + 1>(x, y, z, u, cr, ci, Mg, ez, ez2, epr, epi);
}

__host__ __device__ __forceinline__ float zg_rcp(float x) {
#ifdef __CUDA_ARCH__
  return __frcp_rn(x);
#else
  return 1.0f / x;
#endif
}

// field of a group's expansion at the scaled offset (x, y, z) (|v| > 1)
__host__ __device__ __forceinline__ void zg_multipole(float x, float y, float z,
                                             const float2* __restrict__ Mg, float& fx, float& fy,
                                             float& fz) {
  const float u = zg_rcp(fmaf(x, x, fmaf(y, y, z * z)));
  float ez = 0.f, ez2 = 0.f, epr = 0.f, epi = 0.f;
  zg_cols<0>(x, y, z, u, sqrtf(u), 0.f, Mg, ez, ez2, epr, epi);
  fx = epr;
  fy = epi;
  fz = fmaf(2.f, ez2, ez);
}

// Block = 128 nuclei (in group order) x kZChunk groups.  Partial fields per
// chunk to out[chunk][target][3] (target in group order).
__global__ void __launch_bounds__(kZTile) k_zg_field(int nsph, int ngroup,
                                                     const int* __restrict__ gsph,
                                                     const double4* __restrict__ sph,
                                                     const double4* __restrict__ gcen,
                                                     const int* __restrict__ gptr,
                                                     const float4* __restrict__ zpk,
                                                     const float2* __restrict__ M,
                                                     double* __restrict__ out) {
  __shared__ float2 sM[kZChunk][kZNM];
  __shared__ double4 sC[kZChunk];
  __shared__ int sP[kZChunk + 1];
  __shared__ float4 sT[kZTile / 32][32];  // per-warp point tiles of the direct sums
  const int tid = threadIdx.x, ch = blockIdx.y;
  const int g0 = ch * kZChunk, ng = min(ngroup - g0, kZChunk);
  for (int e = tid; e < ng * kZNM; e += kZTile) sM[e / kZNM][e % kZNM] = M[(size_t)g0 * kZNM + e];
  if (tid < ng) sC[tid] = gcen[g0 + tid];
  if (tid <= ng) sP[tid] = gptr[g0 + tid];
  __syncthreads();
  const int tt = blockIdx.x * kZTile + tid;
  const bool act = tt < nsph;
  const double4 ci = act ? sph[gsph[tt]] : make_double4(0.0, 0.0, 0.0, 0.0);
  double ex = 0.0, ey = 0.0, ez = 0.0;
  for (int gi = 0; gi < ng; ++gi) {
    const double4 cg = sC[gi];
    const double dx = ci.x - cg.x, dy = ci.y - cg.y, dz = ci.z - cg.z;
    const double d2 = dx * dx + dy * dy + dz * dz, rr = kZetaRho * cg.w;
    const bool far = !act || d2 > rr * rr;
    if (__all_sync(kFull, far)) {
      const double ia = 1.0 / cg.w;
      float fx, fy, fz;
      zg_multipole((float)(dx * ia), (float)(dy * ia), (float)(dz * ia), sM[gi], fx, fy, fz);
      const double s = ia * ia;
      ex += (double)fx * s;
      ey += (double)fy * s;
      ez += (double)fz * s;
    } else {
      // the warp's own tiles of 32 points: one coalesced load per lane (the
      // next tile's in flight while this one is summed), broadcast reads
      // from shared memory; the padding of a last partial tile has charge
      // zero and sits far away
      const int w = tid >> 5, lane = tid & 31;
      const float vx = (float)dx, vy = (float)dy, vz = (float)dz;
      const int kb = sP[gi], k1 = sP[gi + 1];
      const float4 pad = make_float4(1e4f, 1e4f, 1e4f, 0.f);
      float4 nxt = kb + lane < k1 ? zpk[kb + lane] : pad;
      float fx = 0.f, fy = 0.f, fz = 0.f;
      int t = 0;
      for (int k0 = kb; k0 < k1; k0 += 32, ++t) {
        __syncwarp();
        sT[w][lane] = nxt;
        __syncwarp();
        const int kn = k0 + 32 + lane;
        nxt = kn < k1 ? zpk[kn] : pad;
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
          const float4 p = sT[w][j];
          const float qx = vx - p.x, qy = vy - p.y, qz = vz - p.z;
          const float r2 = fmaf(qx, qx, fmaf(qy, qy, qz * qz));
          const float ri = rsqrtf(r2);
          const float wv = p.w * (ri * ri * ri);
          fx = fmaf(wv, qx, fx);
          fy = fmaf(wv, qy, fy);
          fz = fmaf(wv, qz, fz);
        }
        if ((t & 7) == 7) {  // FP32 partial sums of 256 points into FP64
          ex += fx;
          ey += fy;
          ez += fz;
          fx = fy = fz = 0.f;
        }
      }
      ex += fx;
      ey += fy;
      ez += fz;
    }
  }
  if (act) {
    double* o = out + ((size_t)ch * nsph + tt) * 3;
    o[0] = ex;
    o[1] = ey;
    o[2] = ez;
  }
}

// ef(3, sphere) = sum over the chunks in order
__global__ void k_zg_reduce(int nsph, int nchunk, const int* __restrict__ gsph,
                            const double* __restrict__ part, double* __restrict__ ef) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3LL * nsph) return;
  const int tt = (int)(e / 3), c = (int)(e % 3);
  double s = 0.0;
  for (int k = 0; k < nchunk; ++k) s += part[((size_t)k * nsph + tt) * 3 + c];
  ef[3 * (size_t)gsph[tt] + c] = s;
}

}  // namespace

size_t zgroups_scan_bytes(int nsph) { return scan_temp_bytes(nsph); }

cudaError_t launch_zgroups_cells(Launch L, int nsph, const double4* sph, ZGroups& zg,
                                 int* dcount, int* hcount) {
  if (nsph <= 0) return cudaErrorInvalidValue;
  k_zg_build<<<1, 1024, 0, L.st>>>(nsph, sph, kZetaCell, zg.cellid, zg.gsph, zg.gstart, dcount);
  ++*L.launches;
  cudaError_t e;
  if ((e = cudaGetLastError())) return e;
  if ((e = cudaMemcpyAsync(hcount, dcount, sizeof(int), cudaMemcpyDeviceToHost, L.st))) return e;
  if ((e = cudaStreamSynchronize(L.st))) return e;
  zg.ngroup = *hcount;
  if (zg.ngroup <= 0 || zg.ngroup > nsph) return cudaErrorUnknown;
  k_zg_geom<<<(zg.ngroup + 3) / 4, 128, 0, L.st>>>(zg.ngroup, zg.gstart, zg.gsph, sph, zg.gcen);
  ++*L.launches;
  return cudaGetLastError();
}

cudaError_t launch_zgroups_points(Launch L, const int* cavoff, ZGroups& zg, void* scan_tmp,
                                  size_t scan_bytes) {
  k_zg_npt<<<(zg.ngroup + 4) / 4, 128, 0, L.st>>>(zg.ngroup, zg.gstart, zg.gsph, cavoff, zg.gnpt);
  ++*L.launches;
  cudaError_t e;
  if ((e = cudaGetLastError())) return e;
  return scan_exclusive(L, zg.gnpt, zg.gptr, zg.ngroup, scan_tmp, scan_bytes);
}

int zgroups_nchunk(const ZGroups& zg) { return (zg.ngroup + kZChunk - 1) / kZChunk; }
size_t zgroups_moment_count(const ZGroups& zg) { return (size_t)zg.ngroup * kZNM; }

cudaError_t launch_zeta_field_far(Launch L, int nsph, const double4* sph, const int* cavoff,
                                  const double* ccav, const double* zeta, const ZGroups& zg,
                                  float4* zpk, float2* M, double* scratch, double* ef) {
  if (nsph == 0) return cudaSuccess;
  k_zg_moments<<<zg.ngroup, 128, 0, L.st>>>(zg.gstart, zg.gsph, zg.gcen, zg.gptr, cavoff, ccav,
                                            zeta, zpk, M);
  ++*L.launches;
  cudaError_t e;
  if ((e = cudaGetLastError())) return e;
  const int nchunk = zgroups_nchunk(zg);
  dim3 grid((nsph + kZTile - 1) / kZTile, nchunk);
  k_zg_field<<<grid, kZTile, 0, L.st>>>(nsph, zg.ngroup, zg.gsph, sph, zg.gcen, zg.gptr, zpk, M,
                                        scratch);
  ++*L.launches;
  if ((e = cudaGetLastError())) return e;
  k_zg_reduce<<<(unsigned)((3LL * nsph + 255) / 256), 256, 0, L.st>>>(nsph, nchunk, zg.gsph,
                                                                      scratch, ef);
  ++*L.launches;
  return cudaGetLastError();
}

}  // namespace ddc
