// ddc_guess.cu -- learned initial guess for the direct and adjoint solves.
//
// The reference starts both Jacobi/DIIS solves from X0 = D^-1 g and
// S0 = D^-1 psi (cosmo.f90:136-138, 174-176).  Here a small per-sphere
// network predicts the correction to that start from the sphere's own data:
//
//   features (per sphere i): its nylm right-hand-side coefficients g_i(lm),
//     the adjoint right-hand side psi_i(00) (= sqrt(4 pi) q_i), its radius and
//     a 16-bin histogram of the distances to the other centres of its
//     molecule (bins of 0.5 angstrom from 0 to 8 angstrom), zero-padded to a
//     multiple of 16 and standardised with the model's stored statistics;
//   network: Linear -> ReLU, three hidden layers of `hidden` units, Linear;
//     weights used in BF16 by every product, FP32 accumulation; FP32 master
//     weights and Adam moments for training;
//   output: the 2*nylm corrections (X0 - D^-1 g, S0 - D^-1 psi), in units of
//     the model's stored per-output scales.
//
// The solver itself is unchanged: from the predicted start it runs the
// reference's Jacobi/DIIS to the same 10^-iconv stop test, so the guess can
// only change the iteration count, never the converged answer.  Training data
// come from the solver: ddc_guess_features / ddc_guess_targets read the last
// energy+force flow of a context (one molecule or a batch).
//
// Kernels: a tiled SIMT GEMM reading BF16 weights (the three products of a
// dense layer: forward, input gradient, weight gradient), bias/ReLU, the
// loss, Adam, and the feature / target / guess kernels.  All reductions have
// a fixed order (no floating-point atomics).
#include <cuda_bf16.h>

#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "ddc_internal.h"

using namespace ddc;

struct ddc_guess {
  int lmax = 0, nylm = 0, hidden = 0, device = 0;
  int nin = 0, nout = 0;  // padded widths
  int dims[5] = {0};      // layer widths: nin, hidden x3, nout
  long long offw[4] = {0}, offb[4] = {0}, nw = 0, np = 0;
  DBuf p32;    // FP32 master parameters: W0..W3 (row-major [out][in]) then b0..b3
  DBuf wbf;    // BF16 copies of W0..W3
  DBuf mom1, mom2;  // Adam moments
  DBuf stats;  // feature mean [nin], feature 1/std [nin], output scale [nout]
  DBuf act, grad, xin, tgt, part;  // training / inference work
  long long work_rows = 0;
  long long step = 0;
  std::string err;
};

namespace {

constexpr int kHistBins = 16;
constexpr double kBohrPerAng = 1.0 / 0.52917721092;  // main.f90:99
constexpr int GT = 64, GK = 16;                        // GEMM tile (rows, cols), k depth

int pad16(int n) { return (n + 15) / 16 * 16; }

// C[m][n] (ldc) = sum_k A(m,k) B(k,n), FP32 accumulation.
//   A(m,k) = TA ? A[k*lda + m] : A[m*lda + k]                  (FP32)
//   B(k,n) = BNK ? B[n*ldb + k] : B[k*ldb + n]                  (BF16 or FP32)
// 64x64 tiles, 256 threads, 4x4 outputs per thread, 16-deep k slabs.
template <bool TA, bool BNK, class TB>
__global__ void __launch_bounds__(256) k_mlp_gemm(int M, int N, int K, const float* __restrict__ A,
                                                  int lda, const TB* __restrict__ B, int ldb,
                                                  float* __restrict__ C, int ldc) {
  __shared__ float As[GK][GT + 4];
  __shared__ float Bs[GK][GT + 4];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += GK) {
#pragma unroll
    for (int u = 0; u < GT * GK / 256; ++u) {
      const int e = tid + u * 256;
      int mm, kk;
      if (TA) { mm = e % GT; kk = e / GT; } else { kk = e % GK; mm = e / GK; }
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? (TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k]) : 0.f;
      int nn, kb;
      if (BNK) { kb = e % GK; nn = e / GK; } else { nn = e % GT; kb = e / GT; }
      const int n = n0 + nn, kg = k0 + kb;
      float bv = 0.f;
      if (n < N && kg < K) {
        if constexpr (sizeof(TB) == 2)
          bv = __bfloat162float(BNK ? B[(size_t)n * ldb + kg] : B[(size_t)kg * ldb + n]);
        else
          bv = BNK ? B[(size_t)n * ldb + kg] : B[(size_t)kg * ldb + n];
      }
      Bs[kb][nn] = bv;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[kk][ty * 4 + r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx * 4 + c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int m = m0 + ty * 4 + r;
    if (m >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int n = n0 + tx * 4 + c;
      if (n < N) C[(size_t)m * ldc + n] = acc[r][c];
    }
  }
}

template <bool TA, bool BNK, class TB>
cudaError_t mlp_gemm(cudaStream_t st, int M, int N, int K, const float* A, int lda, const TB* B,
                     int ldb, float* C, int ldc) {
  if (M == 0 || N == 0) return cudaSuccess;
  dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
  k_mlp_gemm<TA, BNK, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc);
  return cudaGetLastError();
}

// y[r][c] = relu(y[r][c] + b[c]) (relu = false: bias only)
__global__ void k_bias_act(long long rows, int cols, const float* __restrict__ b, float* y,
                           bool relu) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * cols) return;
  float v = y[e] + b[(int)(e % cols)];
  y[e] = relu ? fmaxf(v, 0.f) : v;
}
// dh[e] *= (h[e] > 0)
__global__ void k_relu_bwd(long long n, const float* __restrict__ h, float* dh) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n && !(h[e] > 0.f)) dh[e] = 0.f;
}
// db[c] = sum_r dy[r][c], rows in order (one thread per column)
__global__ void k_colsum(int rows, int cols, const float* __restrict__ dy, float* db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += dy[(size_t)r * cols + c];
  db[c] = s;
}
// standardised input rows: xin[r][k] = (feat[order[r]][k] - mean[k]) * istd[k]
// and scaled targets tgt[r][o] = target[order[r]][o] / scale[o]
__global__ void k_gather_rows(int rows, int nin, int nout, const int* __restrict__ order,
                              long long r0, const float* __restrict__ feat,
                              const float* __restrict__ target, const float* __restrict__ stats,
                              float* xin, float* tgt) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int w = nin + nout;
  if (e >= (long long)rows * w) return;
  const int r = (int)(e / w), k = (int)(e - (long long)r * w);
  const long long src = order ? order[r0 + r] : r0 + r;
  if (k < nin) {
    xin[(size_t)r * nin + k] = (feat[src * nin + k] - stats[k]) * stats[nin + k];
  } else if (target) {
    const int o = k - nin;
    tgt[(size_t)r * nout + o] = target[src * nout + o] / stats[2 * nin + o];
  }
}
// loss partials: per block, sum of (y - t)^2; dy = 2 (y - t) / (rows * nout)
__global__ void k_mse(long long n, float inv, const float* __restrict__ y,
                      const float* __restrict__ t, float* dy, double* partial) {
  __shared__ double sh[256];
  double s = 0.0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const float d = y[e] - t[e];
    dy[e] = 2.f * d * inv;
    s += (double)d * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}
// Adam on the FP32 master parameters; refreshes the BF16 weight copies
__global__ void k_adam(long long np, long long nw, float lr, float b1, float b2, float c1,
                       float c2, float eps, const float* __restrict__ g, float* p, float* m,
                       float* v, __nv_bfloat16* wbf) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np) return;
  const float ge = g[e];
  const float me = b1 * m[e] + (1.f - b1) * ge;
  const float ve = b2 * v[e] + (1.f - b2) * ge * ge;
  m[e] = me;
  v[e] = ve;
  const float pe = p[e] - lr * (me / c1) / (sqrtf(ve / c2) + eps);
  p[e] = pe;
  if (e < nw) wbf[e] = __float2bfloat16(pe);
}
__global__ void k_to_bf16(long long n, const float* __restrict__ x, __nv_bfloat16* y) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) y[e] = __float2bfloat16(x[e]);
}
// column statistics of a [n][cols] matrix: mean and 1/std (std of 0 -> 1);
// rms mode: out[c] = rms (0 -> 1).  One block per column, fixed order.
__global__ void k_colstats(long long n, int cols, const float* __restrict__ x, bool rms,
                           float* out_a, float* out_b) {
  __shared__ double s1[256], s2[256];
  const int c = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (long long r = threadIdx.x; r < n; r += blockDim.x) {
    const double v = x[r * cols + c];
    a += v;
    b += v * v;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s1[threadIdx.x] += s1[threadIdx.x + o];
      s2[threadIdx.x] += s2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double mean = n ? s1[0] / n : 0.0, ms = n ? s2[0] / n : 0.0;
    if (rms) {
      const double r = sqrt(ms);
      out_a[c] = r > 1e-30 ? (float)r : 1.f;
    } else {
      const double var = fmax(ms - mean * mean, 0.0);
      out_a[c] = (float)mean;
      out_b[c] = var > 1e-30 ? (float)(1.0 / sqrt(var)) : 1.f;
    }
  }
}

// raw features of sphere i: g_i (nylm), psi_i(00), r_i, distance histogram
__global__ void k_guess_features(int nsph, int nylm, int nin, const double* __restrict__ g,
                                 const double* __restrict__ psi, const double4* __restrict__ sph,
                                 const int2* __restrict__ mrange, float* feat) {
  __shared__ float4 src[128];
  __shared__ int hist[128][kHistBins + 1];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < nsph;
  const double4 ci = ok ? sph[i] : make_double4(0, 0, 0, 0);
  for (int b = 0; b < kHistBins; ++b) hist[threadIdx.x][b] = 0;
  int lo = 0, hi = nsph;
  // the block's source range covers the molecules of its spheres
  int blo = nsph, bhi = 0;
  {
    const int first = blockIdx.x * blockDim.x;
    const int last = min(nsph, first + (int)blockDim.x) - 1;
    if (mrange) {
      blo = mrange[first].x;
      bhi = mrange[last].y;
      if (ok) {
        lo = mrange[i].x;
        hi = mrange[i].y;
      }
    } else {
      blo = 0;
      bhi = nsph;
    }
  }
  const float bin = (float)(0.5 * kBohrPerAng);
  for (int j0 = blo; j0 < bhi; j0 += blockDim.x) {
    const int j = j0 + threadIdx.x;
    __syncthreads();
    if (j < bhi) {
      const double4 cj = sph[j];
      src[threadIdx.x] = make_float4((float)cj.x, (float)cj.y, (float)cj.z, 0.f);
    }
    __syncthreads();
    const int cnt = min((int)blockDim.x, bhi - j0);
    if (ok) {
      for (int k = 0; k < cnt; ++k) {
        const int jj = j0 + k;
        if (jj < lo || jj >= hi || jj == i) continue;
        const float4 s = src[k];
        const float dx = s.x - (float)ci.x, dy = s.y - (float)ci.y, dz = s.z - (float)ci.z;
        const float d = sqrtf(dx * dx + dy * dy + dz * dz);
        const int b = (int)(d / bin);
        if (b < kHistBins) hist[threadIdx.x][b]++;
      }
    }
  }
  if (!ok) return;
  float* f = feat + (size_t)i * nin;
  for (int k = 0; k < nylm; ++k) f[k] = (float)g[(size_t)i * nylm + k];
  f[nylm] = (float)psi[(size_t)i * nylm];
  f[nylm + 1] = (float)ci.w;
  for (int b = 0; b < kHistBins; ++b) f[nylm + 2 + b] = (float)hist[threadIdx.x][b];
  for (int k = nylm + 2 + kHistBins; k < nin; ++k) f[k] = 0.f;
}

// targets: t[i][lm] = X - facl g, t[i][nylm + lm] = S - facl psi (zero-padded)
__global__ void k_guess_targets(const YlmTables tb, int nsph, int nout,
                                const double* __restrict__ g, const double* __restrict__ psi,
                                const double* __restrict__ X, const double* __restrict__ S,
                                float* t) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)nsph * nout) return;
  const int i = (int)(e / nout), o = (int)(e - (long long)i * nout);
  const int nylm = tb.nylm;
  float v = 0.f;
  if (o < 2 * nylm) {
    const int lm = o % nylm;
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) ++l;
    const size_t q = (size_t)i * nylm + lm;
    v = o < nylm ? (float)(X[q] - tb.facl[l] * g[q]) : (float)(S[q] - tb.facl[l] * psi[q]);
  }
  t[e] = v;
}

// guesses from the network output: x = facl g + scale * out (and s likewise)
__global__ void k_guess_apply(const YlmTables tb, int nsph, int nout,
                              const float* __restrict__ out, const float* __restrict__ scale,
                              const double* __restrict__ g, const double* __restrict__ psi,
                              double* x, double* s) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nylm = tb.nylm;
  if (e >= (long long)nsph * nylm) return;
  const int i = (int)(e / nylm), lm = (int)(e - (long long)i * nylm);
  int l = 0;
  while ((l + 1) * (l + 1) <= lm) ++l;
  const float* o = out + (size_t)i * nout;
  if (x) x[e] = tb.facl[l] * g[e] + (double)(scale[lm] * o[lm]);
  if (s) s[e] = tb.facl[l] * psi[e] + (double)(scale[nylm + lm] * o[nylm + lm]);
}

unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

int gfail(ddc_guess* m, int code, const std::string& msg) {
  if (m) m->err = msg;
  return code;
}
#define GCK(expr)                                                                      \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess) {                                                           \
      cudaGetLastError();                                                              \
      return gfail(m, _e == cudaErrorMemoryAllocation ? DDC_ERR_NOMEM : DDC_ERR_CUDA, \
                   std::string(#expr) + ": " + cudaGetErrorString(_e));               \
    }                                                                                  \
  } while (0)

// work buffers for `rows` rows per pass
int ensure_work(ddc_guess* m, long long rows) {
  if (rows <= m->work_rows) return DDC_OK;
  long long acts = (long long)m->dims[0] + 3LL * m->hidden + m->dims[4];
  GCK(m->act.ensure(sizeof(float) * rows * acts));
  GCK(m->grad.ensure(sizeof(float) * rows * (2LL * m->hidden + m->dims[4])));
  GCK(m->xin.ensure(sizeof(float) * rows * m->nin));
  GCK(m->tgt.ensure(sizeof(float) * rows * m->nout));
  GCK(m->part.ensure(sizeof(double) * 1024));
  m->work_rows = rows;
  return DDC_OK;
}

// activations of layer l (l = 0: the standardised input) for `rows` rows
float* act_ptr(ddc_guess* m, int l, long long rows) {
  float* a = m->act.as<float>();
  long long off = 0;
  for (int k = 0; k < l; ++k) off += (long long)rows * m->dims[k];
  return a + off;
}

// forward pass of `rows` standardised rows already in act layer 0
int forward(ddc_guess* m, cudaStream_t st, int rows) {
  const __nv_bfloat16* wb = m->wbf.as<__nv_bfloat16>();
  const float* b = m->p32.as<float>();
  for (int l = 0; l < 4; ++l) {
    const int din = m->dims[l], dout = m->dims[l + 1];
    float* x = act_ptr(m, l, rows);
    float* y = act_ptr(m, l + 1, rows);
    GCK((mlp_gemm<false, true, __nv_bfloat16>(st, rows, dout, din, x, din, wb + m->offw[l], din,
                                              y, dout)));
    k_bias_act<<<blocks((long long)rows * dout), 256, 0, st>>>(rows, dout, b + m->offb[l], y,
                                                               l < 3);
    GCK(cudaGetLastError());
  }
  return DDC_OK;
}

}  // namespace

extern "C" {

int ddc_guess_create(int lmax, int hidden, int device, ddc_guess** out) {
  if (!out || lmax < 0 || lmax > DDC_MAX_LMAX || hidden < 16 || hidden > 4096 || device < 0)
    return DDC_ERR_PARAM;
  ddc_guess* m = new ddc_guess();
  m->lmax = lmax;
  m->nylm = (lmax + 1) * (lmax + 1);
  m->hidden = pad16(hidden);
  m->device = device;
  m->nin = pad16(m->nylm + 2 + kHistBins);
  m->nout = pad16(2 * m->nylm);
  m->dims[0] = m->nin;
  m->dims[1] = m->dims[2] = m->dims[3] = m->hidden;
  m->dims[4] = m->nout;
  long long o = 0;
  for (int l = 0; l < 4; ++l) {
    m->offw[l] = o;
    o += (long long)m->dims[l] * m->dims[l + 1];
  }
  m->nw = o;
  for (int l = 0; l < 4; ++l) {
    m->offb[l] = o;
    o += m->dims[l + 1];
  }
  m->np = o;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    delete m;
    return DDC_ERR_CUDA;
  }
  int rc = DDC_OK;
  if (m->p32.ensure(sizeof(float) * m->np) || m->wbf.ensure(2 * m->nw) ||
      m->mom1.ensure(sizeof(float) * m->np) || m->mom2.ensure(sizeof(float) * m->np) ||
      m->stats.ensure(sizeof(float) * (2 * m->nin + m->nout)))
    rc = DDC_ERR_NOMEM;
  if (rc == DDC_OK) {
    // default statistics: identity standardisation, unit output scales
    std::vector<float> st(2 * m->nin + m->nout, 1.f);
    for (int k = 0; k < m->nin; ++k) st[k] = 0.f;
    if (cudaMemcpy(m->stats.p, st.data(), sizeof(float) * st.size(), cudaMemcpyHostToDevice) ||
        cudaMemset(m->p32.p, 0, sizeof(float) * m->np) || cudaMemset(m->wbf.p, 0, 2 * m->nw) ||
        cudaMemset(m->mom1.p, 0, sizeof(float) * m->np) ||
        cudaMemset(m->mom2.p, 0, sizeof(float) * m->np))
      rc = DDC_ERR_CUDA;
  }
  if (rc != DDC_OK) {
    cudaGetLastError();
    delete m;
    return rc;
  }
  *out = m;
  return DDC_OK;
}

int ddc_guess_destroy(ddc_guess* m) {
  if (!m) return DDC_ERR_PARAM;
  cudaSetDevice(m->device);
  delete m;
  return DDC_OK;
}

const char* ddc_guess_last_error(ddc_guess* m) { return m ? m->err.c_str() : "null model"; }

int ddc_guess_sizes(ddc_guess* m, int* nfeat, int* nout, long long* nparams) {
  if (!m) return DDC_ERR_PARAM;
  if (nfeat) *nfeat = m->nin;
  if (nout) *nout = m->nout;
  if (nparams) *nparams = m->np + 2LL * m->nin + m->nout;
  return DDC_OK;
}

int ddc_guess_get_params(ddc_guess* m, float* host) {
  if (!m || !host) return DDC_ERR_PARAM;
  cudaSetDevice(m->device);
  GCK(cudaMemcpy(host, m->p32.p, sizeof(float) * m->np, cudaMemcpyDeviceToHost));
  GCK(cudaMemcpy(host + m->np, m->stats.p, sizeof(float) * (2 * m->nin + m->nout),
                 cudaMemcpyDeviceToHost));
  return DDC_OK;
}

int ddc_guess_set_params(ddc_guess* m, const float* host) {
  if (!m || !host) return DDC_ERR_PARAM;
  cudaSetDevice(m->device);
  GCK(cudaMemcpy(m->p32.p, host, sizeof(float) * m->np, cudaMemcpyHostToDevice));
  GCK(cudaMemcpy(m->stats.p, host + m->np, sizeof(float) * (2 * m->nin + m->nout),
                 cudaMemcpyHostToDevice));
  k_to_bf16<<<blocks(m->nw), 256>>>(m->nw, m->p32.as<float>(), m->wbf.as<__nv_bfloat16>());
  GCK(cudaGetLastError());
  GCK(cudaMemset(m->mom1.p, 0, sizeof(float) * m->np));
  GCK(cudaMemset(m->mom2.p, 0, sizeof(float) * m->np));
  m->step = 0;
  GCK(cudaDeviceSynchronize());
  return DDC_OK;
}

int ddc_guess_init_random(ddc_guess* m, unsigned long long seed) {
  if (!m) return DDC_ERR_PARAM;
  // He-uniform weights, zero biases; statistics kept
  std::mt19937_64 rng(seed);
  std::vector<float> p(m->np, 0.f);
  for (int l = 0; l < 4; ++l) {
    const double a = std::sqrt(6.0 / m->dims[l]) * (l == 3 ? 0.1 : 1.0);
    std::uniform_real_distribution<double> u(-a, a);
    for (long long k = 0; k < (long long)m->dims[l] * m->dims[l + 1]; ++k)
      p[m->offw[l] + k] = (float)u(rng);
  }
  std::vector<float> st(2 * m->nin + m->nout);
  cudaSetDevice(m->device);
  GCK(cudaMemcpy(st.data(), m->stats.p, sizeof(float) * st.size(), cudaMemcpyDeviceToHost));
  p.insert(p.end(), st.begin(), st.end());
  return ddc_guess_set_params(m, p.data());
}

int ddc_guess_fit_scaling(ddc_guess* m, const float* feat, const float* target, long long n) {
  if (!m || !feat || !target || n <= 0) return DDC_ERR_PARAM;
  cudaSetDevice(m->device);
  float* st = m->stats.as<float>();
  k_colstats<<<m->nin, 256>>>(n, m->nin, feat, false, st, st + m->nin);
  GCK(cudaGetLastError());
  k_colstats<<<m->nout, 256>>>(n, m->nout, target, true, st + 2 * m->nin, nullptr);
  GCK(cudaGetLastError());
  GCK(cudaDeviceSynchronize());
  return DDC_OK;
}

int ddc_guess_train_epoch(ddc_guess* m, const float* feat, const float* target, const int* order,
                          long long n, int batch, float lr, double* loss) {
  if (!m || !feat || !target || n <= 0 || batch <= 0) return DDC_ERR_PARAM;
  cudaSetDevice(m->device);
  const int rc0 = ensure_work(m, batch);
  if (rc0 != DDC_OK) return rc0;
  cudaStream_t st = nullptr;
  const __nv_bfloat16* wb = m->wbf.as<__nv_bfloat16>();
  DBuf pgrad;  // parameter gradient of one mini-batch
  GCK(pgrad.ensure(sizeof(float) * m->np));
  float* gbuf = pgrad.as<float>();
  const int H = m->hidden, NO = m->nout;
  double total = 0.0;
  long long seen = 0;
  std::vector<double> hp(1024);
  for (long long r0 = 0; r0 < n; r0 += batch) {
    const int rows = (int)std::min<long long>(batch, n - r0);
    k_gather_rows<<<blocks((long long)rows * (m->nin + NO)), 256, 0, st>>>(
        rows, m->nin, NO, order, r0, feat, target, m->stats.as<float>(), act_ptr(m, 0, rows),
        m->tgt.as<float>());
    GCK(cudaGetLastError());
    const int rcf = forward(m, st, rows);
    if (rcf != DDC_OK) return rcf;
    // loss and output gradient
    float* y = act_ptr(m, 4, rows);
    float* dy = m->grad.as<float>();  // [rows][NO], then two [rows][H] buffers
    float* dh0 = dy + (size_t)rows * NO;
    float* dh1 = dh0 + (size_t)rows * H;
    const long long ne = (long long)rows * NO;
    const int nb = (int)std::min<long long>(1024, blocks(ne));
    k_mse<<<nb, 256, 0, st>>>(ne, 1.f / (float)ne, y, m->tgt.as<float>(), dy,
                              m->part.as<double>());
    GCK(cudaGetLastError());
    // backward: layer 3 .. 0
    float* dcur = dy;
    for (int l = 3; l >= 0; --l) {
      const int din = m->dims[l], dout = m->dims[l + 1];
      const float* x = act_ptr(m, l, rows);
      // weight gradient dW[o][i] = sum_r dcur[r][o] x[r][i]
      GCK((mlp_gemm<true, false, float>(st, dout, din, rows, dcur, dout, x, din,
                                        gbuf + m->offw[l], din)));
      k_colsum<<<blocks(dout), 256, 0, st>>>(rows, dout, dcur, gbuf + m->offb[l]);
      GCK(cudaGetLastError());
      if (l > 0) {
        float* dprev = (dcur == dh0) ? dh1 : dh0;
        // input gradient dx[r][i] = sum_o dcur[r][o] W[o][i]
        GCK((mlp_gemm<false, false, __nv_bfloat16>(st, rows, din, dout, dcur, dout,
                                                   wb + m->offw[l], din, dprev, din)));
        k_relu_bwd<<<blocks((long long)rows * din), 256, 0, st>>>((long long)rows * din, x,
                                                                  dprev);
        GCK(cudaGetLastError());
        dcur = dprev;
      }
    }
    ++m->step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    k_adam<<<blocks(m->np), 256, 0, st>>>(m->np, m->nw, lr, b1, b2, c1, c2, 1e-8f, gbuf,
                                          m->p32.as<float>(), m->mom1.as<float>(),
                                          m->mom2.as<float>(), m->wbf.as<__nv_bfloat16>());
    GCK(cudaGetLastError());
    GCK(cudaMemcpyAsync(hp.data(), m->part.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
    GCK(cudaStreamSynchronize(st));
    double s = 0.0;
    for (int k = 0; k < nb; ++k) s += hp[k];
    total += s;
    seen += ne;
  }
  if (loss) *loss = seen ? total / (double)seen : 0.0;
  return DDC_OK;
}

int ddc_guess_predict(ddc_guess* m, const float* feat, float* out, long long n) {
  if (!m || !feat || !out || n < 0) return DDC_ERR_PARAM;
  cudaSetDevice(m->device);
  const int chunk = 65536;
  const int rc0 = ensure_work(m, std::min<long long>(n, chunk));
  if (rc0 != DDC_OK) return rc0;
  for (long long r0 = 0; r0 < n; r0 += chunk) {
    const int rows = (int)std::min<long long>(chunk, n - r0);
    k_gather_rows<<<blocks((long long)rows * (m->nin + m->nout)), 256>>>(
        rows, m->nin, m->nout, nullptr, r0, feat, nullptr, m->stats.as<float>(),
        act_ptr(m, 0, rows), nullptr);
    GCK(cudaGetLastError());
    const int rcf = forward(m, nullptr, rows);
    if (rcf != DDC_OK) return rcf;
    GCK(cudaMemcpyAsync(out + r0 * m->nout, act_ptr(m, 4, rows),
                        sizeof(float) * rows * m->nout, cudaMemcpyDeviceToDevice, nullptr));
  }
  GCK(cudaDeviceSynchronize());
  return DDC_OK;
}

}  // extern "C"

namespace ddc {

int guess_nfeat(const ddc_guess* m) { return m->nin; }
int guess_nout(const ddc_guess* m) { return m->nout; }
int guess_lmax(const ddc_guess* m) { return m->lmax; }

cudaError_t launch_guess_features(Launch L, int nsph, int nylm, int nin, const double* g,
                                  const double* psi, const double4* sph, const int2* mrange,
                                  float* feat) {
  if (nsph == 0) return cudaSuccess;
  k_guess_features<<<blocks(nsph, 128), 128, 0, L.st>>>(nsph, nylm, nin, g, psi, sph, mrange,
                                                         feat);
  ++*L.launches;
  return cudaGetLastError();
}
cudaError_t launch_guess_targets(Launch L, const YlmTables& tb, int nsph, int nout,
                                 const double* g, const double* psi, const double* X,
                                 const double* S, float* t) {
  const long long n = (long long)nsph * nout;
  if (n == 0) return cudaSuccess;
  k_guess_targets<<<blocks(n), 256, 0, L.st>>>(tb, nsph, nout, g, psi, X, S, t);
  ++*L.launches;
  return cudaGetLastError();
}

// Guesses of a context from its features: one inference pass of the model on
// the context's stream, in the model's own activation buffers (grown on
// demand).
cudaError_t guess_infer(Launch L, ddc_guess* m, const YlmTables& tb, int nsph, const float* feat,
                        const double* g, const double* psi, double* x, double* s) {
  if (nsph == 0) return cudaSuccess;
  if (m->work_rows < nsph && ensure_work(m, nsph) != DDC_OK) return cudaErrorMemoryAllocation;
  k_gather_rows<<<blocks((long long)nsph * (m->nin + m->nout)), 256, 0, L.st>>>(
      nsph, m->nin, m->nout, nullptr, 0, feat, nullptr, m->stats.as<float>(), act_ptr(m, 0, nsph),
      nullptr);
  ++*L.launches;
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  const __nv_bfloat16* wb = m->wbf.as<__nv_bfloat16>();
  const float* b = m->p32.as<float>();
  for (int l = 0; l < 4; ++l) {
    const int din = m->dims[l], dout = m->dims[l + 1];
    float* xa = act_ptr(m, l, nsph);
    float* ya = act_ptr(m, l + 1, nsph);
    if ((e = mlp_gemm<false, true, __nv_bfloat16>(L.st, nsph, dout, din, xa, din,
                                                  wb + m->offw[l], din, ya, dout)))
      return e;
    k_bias_act<<<blocks((long long)nsph * dout), 256, 0, L.st>>>(nsph, dout, b + m->offb[l], ya,
                                                                 l < 3);
    *L.launches += 2;
    if ((e = cudaGetLastError())) return e;
  }
  k_guess_apply<<<blocks((long long)nsph * tb.nylm), 256, 0, L.st>>>(
      tb, nsph, m->nout, act_ptr(m, 4, nsph), m->stats.as<float>() + 2 * m->nin, g, psi, x, s);
  ++*L.launches;
  return cudaGetLastError();
}

}  // namespace ddc
