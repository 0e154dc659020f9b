// ddc_tc.cu -- the two dense contractions of every mixed-precision operator
// application, on the fifth-generation tensor cores (tcgen05, sm_100a).
//
//   projection (intrhs inside lx, matvec.f90:131-135; ddcosmo.f90:789-821):
//       y(lm, i) = alpha * sum_n bw(lm, n) pot(n, i)         M = lm, K = n
//   expansion (xi = basis^T s, matvec.f90:189-204):
//       xi(n, i) = sum_lm basis(lm, n) s(lm, i)               M = n,  K = lm
//
// Both run as TF32 tensor-core GEMMs with the three-term split that recovers
// FP32 accuracy: every operand v is carried as hi = tf32(v) and
// lo = tf32(v - hi), and each k-step issues A_hi*B_hi + A_hi*B_lo + A_lo*B_hi
// into one FP32 accumulator in tensor memory (the dropped A_lo*B_lo term and
// the truncation of the lo parts are below 2^-20 of each product).  The
// static operand (bw or basis) is split once, at set-up, from its FP64 values
// into a packed image whose 16 KB chunks are the exact shared-memory tiles the
// MMA reads (K-major, 128-byte swizzle), so a chunk arrives with one bulk copy.
// The per-call operand is split on the way in: the grid field pot (FP32, row
// stride padded to 16 bytes) arrives by a TMA tensor load in the same swizzled
// layout and is split in place; the coefficient vector s (FP64) is read and
// split by the epilogue warps before the MMAs start.  The epilogue widens the
// projection to FP64 with alpha applied (no separate conversion pass) and
// writes xi as FP32 in the layout of the fused L / L* kernel.
//
// Roles (one CTA per output tile -- for the expansion, one 128-point grid
// tile of one group of spheres -- 10 warps):
//   warp 0      one lane issues the bulk / TMA copies into a ring of stages
//   warp 1      allocates tensor memory; one lane issues the MMAs
//   warps 2..9  split the per-call operand, then drain the accumulator
// Every wait on an mbarrier is bounded (2 s of %globaltimer); a wait that runs
// out sets the caller's error flag and the CTA unwinds: the producer waits
// (bounded) for its copies in flight, the MMA lane commits and waits for its
// MMAs, and tensor memory is freed before the CTA exits.
#include <cuda.h>  // CUtensorMap

#include <algorithm>
#include <vector>

#include "ddc_internal.h"

namespace ddc {
namespace {

constexpr int kTcWarps = 10;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr int kSplitWarps = kTcWarps - 2;
constexpr int kChunk = 16384;           // one 128-row x 128-byte swizzled operand chunk
constexpr int kSmemCap = 227 * 1024;    // opt-in shared memory per CTA
constexpr int kSmemSlack = 1024 + 512;  // 1024-byte alignment + barriers
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of `parity` to complete, for at most kWaitNs.  Gives up
// early when another thread of the CTA has already given up (abort set).
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort, int* err,
                          int code) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  for (;;) {
    if (mbar_try(bar, parity)) return true;
    if (*abort) return false;
    if (gtimer() - t0 > kWaitNs) {
      *abort = 1;
      atomicExch(err, code);
      return false;
    }
  }
}
// Bounded wait used while unwinding: ignores the abort flag.
__device__ void mbar_drain(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = gtimer();
  while (!mbar_try(bar, parity))
    if (gtimer() - t0 > kWaitNs) return;
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 1-D bulk copy global -> shared, completion counted on `bar`
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
// 2-D TMA tile load (x = innermost coordinate, in elements)
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, both K-major, TF32 in, FP32 accumulate
__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on `bar` once every MMA issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns of tensor memory
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// Shared-memory descriptor of a K-major operand tile with the 128-byte
// swizzle: rows of 128 bytes (32 TF32 values along K), 8-row groups 1024
// bytes apart.  Fields: start address >> 4 (bits 0-13), leading byte offset
// (unused for this layout, 16 bytes), stride byte offset 1024 >> 4 (bits
// 32-45), descriptor version 1 (bits 46-47), swizzle mode 2 = 128 B (61-63).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), A and
// B TF32 (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at 24.
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}
// Byte offset of element (row r, k) of a swizzled 128-byte-row tile (k < 32).
__device__ __forceinline__ uint32_t sw128_off(int r, int k) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 2) ^ (r & 7)) & 7) << 4) +
                    ((k & 3) << 2));
}
__device__ __forceinline__ float tf32_rna(float v) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
  return __uint_as_float(h);
}
// v = hi + lo with hi, lo TF32 values (|v - hi - lo| <= 2^-21 |v|)
__device__ __forceinline__ void split_f32(float v, float& hi, float& lo) {
  hi = tf32_rna(v);
  lo = tf32_rna(v - hi);
}
__device__ __forceinline__ void split_f64(double v, float& hi, float& lo) {
  hi = tf32_rna((float)v);
  lo = tf32_rna((float)(v - (double)hi));
}

__host__ __device__ constexpr uint32_t tmem_cols(int n) {
  return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : n <= 256 ? 256u : 512u;
}

// ---------------------------------------------------------------------------
// packed image of a static operand: A(m, k) for m < M, k < K (zero beyond),
// chunk (mt, kc) at ((mt*KC + kc)*2 + part) * kChunk bytes, part 0 = hi, 1 = lo.
// src is [G][Y] FP64 (basis or bw): trans = false reads A(m, k) = src[k*ld + m]
// (projection: m = lm, k = grid point), trans = true reads src[m*ld + k]
// (expansion: m = grid point, k = lm).
// ---------------------------------------------------------------------------
__global__ void k_pack_static(const double* __restrict__ src, int ld, bool trans, int M, int K,
                              int MT, int KC, float* img) {
  const long long total = (long long)MT * KC * 128 * 32;
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int k32 = (int)(e & 31), r = (int)((e >> 5) & 127);
  const long long ch = e >> 12;  // (mt*KC + kc)
  const int kc = (int)(ch % KC), mt = (int)(ch / KC);
  const int m = mt * 128 + r, k = kc * 32 + k32;
  double v = 0.0;
  if (m < M && k < K) v = trans ? src[(size_t)m * ld + k] : src[(size_t)k * ld + m];
  float hi, lo;
  split_f64(v, hi, lo);
  unsigned char* base = reinterpret_cast<unsigned char*>(img) + (size_t)ch * 2 * kChunk;
  *reinterpret_cast<float*>(base + sw128_off(r, k32)) = hi;
  *reinterpret_cast<float*>(base + kChunk + sw128_off(r, k32)) = lo;
}

// Accumulation.  The tensor cores round a sum toward zero each time an MMA
// adds into its accumulator, so a long K loop in one accumulator drifts (a
// bias of up to 2^-23 of the partial per step: 4-5e-6 of the result over the
// 590-point projection).  Both kernels therefore keep two accumulators per
// tile (after Ootomo and Yokota, "Recovering single precision accuracy from
// Tensor Cores while surpassing the FP32 theoretical peak performance", 2022):
//   * the main term A_hi*B_hi of one 32-wide K chunk (four MMAs) goes into a
//     fresh accumulator, which the epilogue warps add into FP32 registers
//     (round to nearest) before the MMAs of chunk + 2 reuse it (ping-pong);
//   * the correction terms A_hi*B_lo + A_lo*B_hi, 2^-11 of the main term,
//     stay in one accumulator over the whole K loop (their rounding is
//     negligible) and are added at the end.
// Tensor memory: columns [0, bn) and [bn, 2 bn) hold the two main buffers,
// [2 bn, 3 bn) the correction.  The epilogue thread (lane quarter q of the
// 128 rows, column half h) owns columns 16 h + 32 j, j < kMaxJ.
constexpr int kMaxJ = 5;             // bn <= 32 * kMaxJ = 160
constexpr int kMaxBn = 32 * kMaxJ;

// acc[16 j + k] += tensor memory (rows 32 q.., columns col0 + 16 h + 32 j + k)
__device__ __forceinline__ void tmem_add(uint32_t tmem, int q, int half, uint32_t col0, int bn,
                                         float (&acc)[16 * kMaxJ]) {
#pragma unroll
  for (int j = 0; j < kMaxJ; ++j) {
    const int c = 16 * half + 32 * j;
    if (c < bn) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + col0 + (uint32_t)c, v);
#pragma unroll
      for (int k = 0; k < 16; ++k) acc[16 * j + k] += v[k];
    }
  }
}

// ---------------------------------------------------------------------------
// projection: y(lm, i) = alpha sum_n bw(lm, n) pot(n, i), FP64 out
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTcThreads, 1)
    k_proj_tc(const __grid_constant__ CUtensorMap tm_pot, const float* __restrict__ aimg,
              int nsph, int nylm, int kcn, int bn, int nstage, int nbuf, double alpha,
              double* __restrict__ y, int* err, const SweepMask act) {
  // a batched sweep leaves the tiles of stopped molecules alone (before any
  // barrier or tensor memory is set up)
  if (sweep_skip_tile(act, blockIdx.x * bn, bn, nsph)) return;
  extern __shared__ unsigned char sm_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t bbytes = (uint32_t)bn * 128;
  const uint32_t sbytes = 2 * kChunk + 2 * bbytes;  // A hi | A lo | B hi | B lo
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + (size_t)nstage * sbytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 3 * nstage + 9);
  volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i0 = blockIdx.x * bn;
  const uint32_t sbase = su32(sm);
  const uint32_t bar0 = su32(bars);
  auto FULL = [&](int s) { return bar0 + 8u * s; };
  auto READY = [&](int s) { return bar0 + 8u * (nstage + s); };
  auto EMPTY = [&](int s) { return bar0 + 8u * (2 * nstage + s); };
  auto MFULL = [&](int b) { return bar0 + 8u * (3 * nstage + b); };
  auto MEMPTY = [&](int b) { return bar0 + 8u * (3 * nstage + 4 + b); };
  const uint32_t DONE = bar0 + 8u * (3 * nstage + 8);
  if (threadIdx.x == 0) {
    for (int s = 0; s < nstage; ++s) {
      mbar_init(FULL(s), 1);
      mbar_init(READY(s), kSplitWarps);
      mbar_init(EMPTY(s), 1);
    }
    for (int b = 0; b < nbuf; ++b) {
      mbar_init(MFULL(b), 1);
      mbar_init(MEMPTY(b), kSplitWarps);
    }
    mbar_init(DONE, 1);
    *abort = 0;
    fence_barrier_init();
  }
  const uint32_t ncols = tmem_cols((nbuf + 1) * bn);
  if (warp == 1) tmem_alloc(su32(tslot), ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t corr = tmem + (uint32_t)(nbuf * bn);

  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int kc = 0; kc < kcn; ++kc) {
        const int s = kc % nstage;
        const uint32_t ph = (uint32_t)(kc / nstage) & 1u;
        if (kc >= nstage && !mbar_wait(EMPTY(s), ph ^ 1u, abort, err, 1)) break;
        const uint32_t st = sbase + s * sbytes;
        mbar_expect_tx(FULL(s), 2 * kChunk + bbytes);
        bulk_load(st, aimg + (size_t)kc * (2 * kChunk / 4), 2 * kChunk, FULL(s));
        tma_load_2d(st + 2 * kChunk, &tm_pot, kc * 32, i0, FULL(s));
        issued = kc + 1;
      }
      // copies still in flight land before the CTA exits
      for (int kc = max(0, issued - nstage); kc < issued; ++kc)
        mbar_drain(FULL(kc % nstage), (uint32_t)(kc / nstage) & 1u);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(128, bn);
      for (int kc = 0; kc < kcn; ++kc) {
        const int s = kc % nstage, b = kc % nbuf;
        const uint32_t ph = (uint32_t)(kc / nstage) & 1u;
        if (!mbar_wait(READY(s), ph, abort, err, 2)) break;
        if (kc >= nbuf && !mbar_wait(MEMPTY(b), (uint32_t)(kc / nbuf - 1) & 1u, abort, err, 5))
          break;
        tc_fence_after();
        const uint32_t st = sbase + s * sbytes;
        const uint64_t ah = sw128_desc(st), al = sw128_desc(st + kChunk);
        const uint64_t bh = sw128_desc(st + 2 * kChunk), bl = sw128_desc(st + 2 * kChunk + bbytes);
        const uint32_t mainb = tmem + (uint32_t)(b * bn);
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const uint64_t o = (uint64_t)(ks * 2);  // 32 bytes along K, in 16-byte units
          mma_tf32(mainb, ah + o, bh + o, idesc, ks != 0);
          mma_tf32(corr, ah + o, bl + o, idesc, (kc | ks) != 0);
          mma_tf32(corr, al + o, bh + o, idesc, 1);
        }
        mma_commit(EMPTY(s));
        mma_commit(MFULL(b));
      }
      mma_commit(DONE);
    }
  } else {
    const int t = threadIdx.x - 64;
    const int q = warp & 3, half = (warp - 2) >> 2;
    float acc[16 * kMaxJ];
#pragma unroll
    for (int k = 0; k < 16 * kMaxJ; ++k) acc[k] = 0.f;
    bool ok = true;
    // split chunk kc, then add the main term of chunk kc - lag: up to nbuf
    // chunks' MMAs run while the epilogue works
    const int lag = nbuf - 1;
    for (int kc = 0; ok && kc < kcn + lag; ++kc) {
      if (kc < kcn) {
        const int s = kc % nstage;
        const uint32_t ph = (uint32_t)(kc / nstage) & 1u;
        if (!mbar_wait(FULL(s), ph, abort, err, 3)) {
          ok = false;
          break;
        }
        float4* bh = reinterpret_cast<float4*>(sm + (size_t)s * sbytes + 2 * kChunk);
        float4* bl = reinterpret_cast<float4*>(sm + (size_t)s * sbytes + 2 * kChunk + bbytes);
        for (int e = t; e < (int)(bbytes / 16); e += 32 * kSplitWarps) {
          const float4 v = bh[e];
          float4 h, l;
          split_f32(v.x, h.x, l.x);
          split_f32(v.y, h.y, l.y);
          split_f32(v.z, h.z, l.z);
          split_f32(v.w, h.w, l.w);
          bh[e] = h;
          bl[e] = l;
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(READY(s));
      }
      if (kc >= lag) {
        const int c = kc - lag, b = c % nbuf;
        if (!mbar_wait(MFULL(b), (uint32_t)(c / nbuf) & 1u, abort, err, 4)) {
          ok = false;
          break;
        }
        tc_fence_after();
        tmem_add(tmem, q, half, (uint32_t)(b * bn), bn, acc);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(MEMPTY(b));
      }
    }
    if (ok && mbar_wait(DONE, 0, abort, err, 6)) {
      tc_fence_after();
      tmem_add(tmem, q, half, (uint32_t)(nbuf * bn), bn, acc);
      const int lm = 32 * q + lane;
      if (lm < nylm) {
#pragma unroll
        for (int j = 0; j < kMaxJ; ++j)
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const int i = i0 + 16 * half + 32 * j + k;
            if (16 * half + 32 * j < bn && i < nsph)
              y[(size_t)i * nylm + lm] = alpha * (double)acc[16 * j + k];
          }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    if (*abort && lane == 0) mbar_drain(DONE, 0);  // MMAs issued before giving up
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, ncols);
  }
}

// ---------------------------------------------------------------------------
// expansion: xi(n, i) = sum_lm basis(lm, n) s(lm, i), FP32 out (ld = ngrid)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTcThreads, 1)
    k_xi_tc(const double* __restrict__ s, const float* __restrict__ aimg, int nsph, int nylm,
            int ngrid, int mtn, int mtper, int kcn, int bn, int nstage, float* __restrict__ xi,
            int* err, const SweepMask act) {
  if (sweep_skip_tile(act, blockIdx.x * bn, bn, nsph)) return;
  // this CTA: grid-point tiles mt0 .. mt0 + mtc - 1 (of mtn) for spheres
  // i0 .. i0 + bn (all tiles in one CTA, or one tile per CTA)
  const int mt0 = blockIdx.y * mtper;
  const int mtc = min(mtper, mtn - mt0);
  extern __shared__ unsigned char sm_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t bbytes = (uint32_t)bn * 128;
  unsigned char* bsm = sm;                                   // kcn x (B hi | B lo)
  unsigned char* asm_ = sm + (size_t)kcn * 2 * bbytes;       // nstage x (A hi | A lo)
  uint64_t* bars = reinterpret_cast<uint64_t*>(asm_ + (size_t)nstage * 2 * kChunk);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * nstage + 8);
  volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i0 = blockIdx.x * bn;
  const uint32_t bar0 = su32(bars);
  auto FULL = [&](int st) { return bar0 + 8u * st; };
  auto EMPTY = [&](int st) { return bar0 + 8u * (nstage + st); };
  const uint32_t BREADY = bar0 + 8u * (2 * nstage);
  auto MFULL = [&](int b) { return bar0 + 8u * (2 * nstage + 1 + b); };
  auto MEMPTY = [&](int b) { return bar0 + 8u * (2 * nstage + 3 + b); };
  const uint32_t CFULL = bar0 + 8u * (2 * nstage + 5);
  const uint32_t CEMPTY = bar0 + 8u * (2 * nstage + 6);
  const uint32_t DONE = bar0 + 8u * (2 * nstage + 7);
  if (threadIdx.x == 0) {
    for (int st = 0; st < nstage; ++st) {
      mbar_init(FULL(st), 1);
      mbar_init(EMPTY(st), 1);
    }
    mbar_init(BREADY, kSplitWarps);
    for (int b = 0; b < 2; ++b) {
      mbar_init(MFULL(b), 1);
      mbar_init(MEMPTY(b), kSplitWarps);
    }
    mbar_init(CFULL, 1);
    mbar_init(CEMPTY, kSplitWarps);
    mbar_init(DONE, 1);
    *abort = 0;
    fence_barrier_init();
  }
  const uint32_t ncols = tmem_cols(3 * bn);
  if (warp == 1) tmem_alloc(su32(tslot), ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t corr = tmem + (uint32_t)(2 * bn);
  const int nit = mtc * kcn;

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t abase = su32(asm_);
      int issued = 0;
      for (int it = 0; it < nit; ++it) {
        const int st = it % nstage;
        const uint32_t ph = (uint32_t)(it / nstage) & 1u;
        if (it >= nstage && !mbar_wait(EMPTY(st), ph ^ 1u, abort, err, 11)) break;
        mbar_expect_tx(FULL(st), 2 * kChunk);
        bulk_load(abase + st * 2 * kChunk, aimg + (size_t)(mt0 * kcn + it) * (2 * kChunk / 4),
                  2 * kChunk, FULL(st));
        issued = it + 1;
      }
      for (int it = max(0, issued - nstage); it < issued; ++it)
        mbar_drain(FULL(it % nstage), (uint32_t)(it / nstage) & 1u);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(128, bn);
      const uint32_t abase = su32(asm_), bbase = su32(bsm);
      bool ok = mbar_wait(BREADY, 0, abort, err, 12);
      for (int it = 0; ok && it < nit; ++it) {
        const int mt = it / kcn, kc = it - mt * kcn, st = it % nstage, b = it & 1;
        if (!mbar_wait(FULL(st), (uint32_t)(it / nstage) & 1u, abort, err, 14)) break;
        if (it >= 2 && !mbar_wait(MEMPTY(b), (uint32_t)((it >> 1) - 1) & 1u, abort, err, 13))
          break;
        // the correction accumulator of the previous grid tile has been read
        if (kc == 0 && mt >= 1 && !mbar_wait(CEMPTY, (uint32_t)(mt - 1) & 1u, abort, err, 16))
          break;
        tc_fence_after();
        const uint64_t ah = sw128_desc(abase + st * 2 * kChunk);
        const uint64_t al = sw128_desc(abase + st * 2 * kChunk + kChunk);
        const uint64_t bh = sw128_desc(bbase + kc * 2 * bbytes);
        const uint64_t bl = sw128_desc(bbase + kc * 2 * bbytes + bbytes);
        const uint32_t mainb = tmem + (uint32_t)(b * bn);
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const uint64_t o = (uint64_t)(ks * 2);
          mma_tf32(mainb, ah + o, bh + o, idesc, ks != 0);
          mma_tf32(corr, ah + o, bl + o, idesc, (kc | ks) != 0);
          mma_tf32(corr, al + o, bh + o, idesc, 1);
        }
        mma_commit(EMPTY(st));
        mma_commit(MFULL(b));
        if (kc == kcn - 1) mma_commit(CFULL);
      }
      mma_commit(DONE);  // completes once every MMA issued above has
    }
  } else {
    // split s into the swizzled B tiles: row r = sphere i0 + r, k = lm
    const int t = threadIdx.x - 64;
    const int kp = kcn * 32;
    const int tot = bn * kp;
    constexpr int U = 8;
    for (int e0 = t; e0 < tot; e0 += 32 * kSplitWarps * U) {
      double v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = e0 + u * 32 * kSplitWarps;
        const int r = e / kp, k = e - r * kp;
        v[u] = (e < tot && k < nylm && i0 + r < nsph) ? s[(size_t)(i0 + r) * nylm + k] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = e0 + u * 32 * kSplitWarps;
        if (e < tot) {
          const int r = e / kp, k = e - r * kp;
          float hi, lo;
          split_f64(v[u], hi, lo);
          unsigned char* tile = bsm + (size_t)(k >> 5) * 2 * bbytes;
          const uint32_t o = sw128_off(r, k & 31);
          *reinterpret_cast<float*>(tile + o) = hi;
          *reinterpret_cast<float*>(tile + bbytes + o) = lo;
        }
      }
    }
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) mbar_arrive(BREADY);
    const int q = warp & 3, half = (warp - 2) >> 2;
    float acc[16 * kMaxJ];
#pragma unroll
    for (int k = 0; k < 16 * kMaxJ; ++k) acc[k] = 0.f;
    for (int it = 0; it < nit; ++it) {
      const int mt = it / kcn, kc = it - mt * kcn, b = it & 1;
      if (!mbar_wait(MFULL(b), (uint32_t)(it >> 1) & 1u, abort, err, 15)) break;
      tc_fence_after();
      tmem_add(tmem, q, half, (uint32_t)(b * bn), bn, acc);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(MEMPTY(b));
      if (kc == kcn - 1) {
        if (!mbar_wait(CFULL, (uint32_t)mt & 1u, abort, err, 17)) break;
        tc_fence_after();
        tmem_add(tmem, q, half, (uint32_t)(2 * bn), bn, acc);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(CEMPTY);
        const int m = (mt0 + mt) * 128 + 32 * q + lane;
#pragma unroll
        for (int j = 0; j < kMaxJ; ++j)
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const int i = i0 + 16 * half + 32 * j + k;
            if (m < ngrid && 16 * half + 32 * j < bn && i < nsph)
              xi[(size_t)i * ngrid + m] = acc[16 * j + k];
            acc[16 * j + k] = 0.f;
          }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    if (*abort && lane == 0) mbar_drain(DONE, 0);
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, ncols);
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

// tile width (spheres per CTA): about one tile per SM, a multiple of 16
// (the MMA's N step), at most `cap`
int pick_bn(int nsph, int cap) {
  int want = (nsph + 147) / 148;
  want = ((want + 31) / 32) * 32;
  return std::max(32, std::min(cap, want));
}

}  // namespace

bool tc_supported(int nylm) { return nylm <= 128; }

namespace {

// tile width bn of the projection: pipeline depth, shared memory and the TMA
// box of the grid field (bn rows of 32 values)
cudaError_t cfg_proj(TcPlan& p, int bn) {
  if (bn % 32 != 0 || bn > kMaxBn) return cudaErrorInvalidValue;
  const int sb = 2 * kChunk + 2 * bn * 128;
  p.bn_proj = bn;
  p.ns_proj = std::min(4, (kSmemCap - kSmemSlack) / sb);
  if (p.ns_proj < 2) return cudaErrorInvalidValue;
  // at least 120 KB: one CTA per SM, so tensor-memory allocations never wait
  p.smem_proj = std::max(p.ns_proj * sb + kSmemSlack, 120 * 1024);
  cuuint64_t dims[2] = {(cuuint64_t)p.ngrid, (cuuint64_t)p.nsph};
  cuuint64_t strides[1] = {(cuuint64_t)p.ldp * 4};
  cuuint32_t box[2] = {32, (cuuint32_t)bn};
  cuuint32_t es[2] = {1, 1};
  CUresult r = encode_fn()(&p.tm_pot, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, p.pot_f, dims, strides,
                           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(k_proj_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              p.smem_proj);
}
// tile width of the expansion: the split coefficients of bn spheres stay
// resident, the basis chunks stream through a ring of at least two stages
cudaError_t cfg_xi(TcPlan& p, int bn) {
  if (bn % 32 != 0 || bn > kMaxBn) return cudaErrorInvalidValue;
  const int bsz = p.kc_xi * 2 * bn * 128;
  const int ns = std::min(3, (kSmemCap - kSmemSlack - bsz) / (2 * kChunk));
  if (ns < 2) return cudaErrorInvalidValue;
  p.bn_xi = bn;
  p.ns_xi = ns;
  p.smem_xi = std::max(bsz + ns * 2 * kChunk + kSmemSlack, 120 * 1024);
  return cudaFuncSetAttribute(k_xi_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, p.smem_xi);
}
std::vector<int> bn_candidates(int nsph) {
  std::vector<int> c;
  const int top = std::min(kMaxBn, std::max(32, (nsph + 31) / 32 * 32));
  for (int bn : {pick_bn(nsph, kMaxBn), 32, 64, 96, 128, 160})
    if (bn <= top && std::find(c.begin(), c.end(), bn) == c.end()) c.push_back(bn);
  return c;
}

}  // namespace

cudaError_t tc_plan(Launch L, TcPlan& p, const double* basis, const double* bw, int nsph,
                    int nylm, int ngrid, float* pot_f, int ldp) {
  p.on = false;
  if (!tc_supported(nylm) || nsph <= 0) return cudaSuccess;
  if (!encode_fn()) return cudaErrorNotSupported;
  // the per-call grid field: [nsph][ngrid] FP32 rows ldp apart (16-byte multiple)
  if ((ldp * 4) % 16 != 0 || (reinterpret_cast<uintptr_t>(pot_f) & 15) != 0)
    return cudaErrorInvalidValue;
  p.nsph = nsph;
  p.nylm = nylm;
  p.ngrid = ngrid;
  p.pot_f = pot_f;
  p.ldp = ldp;
  p.kc_proj = (ngrid + 31) / 32;           // projection: M = lm, K = grid points
  p.mt_xi = (ngrid + 127) / 128;           // expansion: M = grid points, K = lm
  p.kc_xi = (nylm + 31) / 32;
  cudaError_t e;
  // default tile widths: about one tile per SM (narrower where the shared
  // memory of a wide tile does not fit)
  int bn = pick_bn(nsph, kMaxBn);
  while ((e = cfg_proj(p, bn)) == cudaErrorInvalidValue && bn > 32) bn -= 32;
  if (e) return e;
  bn = pick_bn(nsph, kMaxBn);
  while ((e = cfg_xi(p, bn)) == cudaErrorInvalidValue && bn > 32) bn -= 32;
  if (e) return e;
  // static operands, split once
  if ((e = p.img_proj.ensure((size_t)p.kc_proj * 2 * kChunk))) return e;
  if ((e = p.img_xi.ensure((size_t)p.mt_xi * p.kc_xi * 2 * kChunk))) return e;
  {
    const long long tot = (long long)p.kc_proj * 128 * 32;
    k_pack_static<<<(unsigned)((tot + 255) / 256), 256, 0, L.st>>>(
        bw, nylm, false, nylm, ngrid, 1, p.kc_proj, p.img_proj.as<float>());
    ++*L.launches;
    const long long tot2 = (long long)p.mt_xi * p.kc_xi * 128 * 32;
    k_pack_static<<<(unsigned)((tot2 + 255) / 256), 256, 0, L.st>>>(
        basis, nylm, true, ngrid, nylm, p.mt_xi, p.kc_xi, p.img_xi.as<float>());
    ++*L.launches;
    if ((e = cudaGetLastError())) return e;
  }
  if (!p.err_h) {
    if ((e = cudaHostAlloc(&p.err_h, sizeof(int), cudaHostAllocMapped))) return e;
    if ((e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&p.err_d), p.err_h, 0))) return e;
  }
  *p.err_h = 0;
  p.on = true;
  return cudaSuccess;
}

// Tile widths picked by measurement: every candidate width of each kernel is
// launched on the context's own buffers (pot_f and s zeroed first; y and xi
// are scratch here) and timed with CUDA events on the context's stream; the
// fastest is kept.  Runs once per problem shape (nsph, nylm, ngrid).
cudaError_t tc_autotune(Launch L, TcPlan& p, const double* s, double* y, float* xi) {
  if (!p.on) return cudaSuccess;
  const long long key = ((long long)p.nsph << 24) ^ ((long long)p.nylm << 12) ^ p.ngrid;
  if (p.tuned && p.tune_key == key) {  // same shape as the last measurement
    p.xi_split = p.tuned_xi_split;
    cudaError_t e = cfg_proj(p, p.tuned_bn_proj);
    return e ? e : cfg_xi(p, p.tuned_bn_xi);
  }
  cudaEvent_t e0, e1;
  cudaError_t e;
  if ((e = cudaEventCreate(&e0))) return e;
  if ((e = cudaEventCreate(&e1))) {
    cudaEventDestroy(e0);
    return e;
  }
  auto timed = [&](auto launch, float* ms) -> cudaError_t {
    cudaError_t r;
    if ((r = launch())) return r;  // warm-up
    if ((r = cudaEventRecord(e0, L.st))) return r;
    for (int k = 0; k < 3; ++k)
      if ((r = launch())) return r;
    if ((r = cudaEventRecord(e1, L.st))) return r;
    if ((r = cudaEventSynchronize(e1))) return r;
    if (p.err_h && *p.err_h) return cudaErrorLaunchFailure;
    return cudaEventElapsedTime(ms, e0, e1);
  };
  const std::vector<int> cand = bn_candidates(p.nsph);
  int best = p.bn_proj;
  float tbest = 1e30f;
  e = cudaMemsetAsync(p.pot_f, 0, sizeof(float) * (size_t)p.nsph * p.ldp, L.st);
  for (size_t k = 0; !e && k < cand.size(); ++k) {
    if (cfg_proj(p, cand[k]) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    float ms = 0.f;
    e = timed([&] { return launch_proj_tc(L, p, 1.0, y); }, &ms);
    if (!e && ms < tbest) {
      tbest = ms;
      best = cand[k];
    }
  }
  if (!e) e = cfg_proj(p, best);
  p.ms_proj = tbest / 3.f;
  best = p.bn_xi;
  bool best_split = false;
  tbest = 1e30f;
  if (!e) e = cudaMemsetAsync(const_cast<double*>(s), 0, sizeof(double) * p.nsph * p.nylm, L.st);
  for (size_t k = 0; !e && k < cand.size(); ++k) {
    if (cfg_xi(p, cand[k]) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    for (int split = 0; !e && split < 2; ++split) {  // all grid tiles per CTA, or one
      p.xi_split = split == 1;
      float ms = 0.f;
      e = timed([&] { return launch_xi_tc(L, p, s, xi); }, &ms);
      if (!e && ms < tbest) {
        tbest = ms;
        best = cand[k];
        best_split = p.xi_split;
      }
    }
  }
  p.xi_split = best_split;
  if (!e) e = cfg_xi(p, best);
  p.ms_xi = tbest / 3.f;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!e) {
    p.tuned = true;
    p.tune_key = key;
    p.tuned_bn_proj = p.bn_proj;
    p.tuned_bn_xi = p.bn_xi;
    p.tuned_xi_split = p.xi_split;
  }
  return e;
}

cudaError_t launch_proj_tc(Launch L, const TcPlan& p, double alpha, double* y,
                           const SweepMask& act) {
  const int grid = (p.nsph + p.bn_proj - 1) / p.bn_proj;
  // main-term buffers in tensor memory: as many as fit beside the correction
  const int nbuf = std::min(4, 512 / p.bn_proj - 1);
  k_proj_tc<<<grid, kTcThreads, p.smem_proj, L.st>>>(p.tm_pot, p.img_proj.as<float>(), p.nsph,
                                                     p.nylm, p.kc_proj, p.bn_proj, p.ns_proj,
                                                     nbuf, alpha, y, p.err_d, act);
  ++*L.launches;
  return cudaGetLastError();
}

cudaError_t launch_xi_tc(Launch L, const TcPlan& p, const double* s, float* xi,
                         const SweepMask& act) {
  const int mtper = p.xi_split ? 1 : p.mt_xi;
  const dim3 grid((p.nsph + p.bn_xi - 1) / p.bn_xi, (p.mt_xi + mtper - 1) / mtper);
  k_xi_tc<<<grid, kTcThreads, p.smem_xi, L.st>>>(s, p.img_xi.as<float>(), p.nsph, p.nylm,
                                                 p.ngrid, p.mt_xi, mtper, p.kc_xi, p.bn_xi,
                                                 p.ns_xi, xi, p.err_d, act);
  ++*L.launches;
  return cudaGetLastError();
}

void tc_release(TcPlan& p) {
  if (p.err_h) cudaFreeHost(p.err_h);
  p.err_h = nullptr;
  p.err_d = nullptr;
  p.on = false;
}

}  // namespace ddc
