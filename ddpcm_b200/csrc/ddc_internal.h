// ddc_internal.h -- shared declarations of the B200 ddCOSMO library.
//
// Layout in HBM (one molecule per context, sizes for N spheres, G grid
// points, Y = (lmax+1)^2 harmonics, P neighbour pairs, T triples):
//   sph[N]         double4 {x, y, z, r} (bohr)
//   grid[G]        double4 {sx, sy, sz, w} (unit vectors, 4pi-scaled weights)
//   basis[G][Y]    Y_lm(s_n); bw[G][Y] = basis * w  (the intrhs operator)
//   inl[N+1], nl[P]      CSR neighbour list, 0-based, ascending j (ddinit)
//   rev[P]               index of (j,i) for the entry (i,j)
//   fi, ui[N][G]         overlap count f_i(n) and cavity weight U_i(n)
//   zi[N][G][3]          grad f (forces only)
//   pn_ptr[P+1], pn[T]   per pair (i,j): grid points n of sphere i with
//                        t_n^ij < 1 (point inside sphere j), ascending n
//   ls_ptr[N+1], ls[T]   per sphere i: (j, n) for j in N_i (CSR order) and the
//                        points n of sphere j inside sphere i (adjoint gather)
//   ntri[N][G]           number of neighbours containing point (i,n)
//   cavoff[N+1], cavidx[N][G], cavpt[ncav], ccav[ncav][3]
// Vectors X(nylm,nsph) live as X[i*nylm + lm], like the reference.
#pragma once
#include <cuda.h>  // CUtensorMap (type only; the driver is reached through cudart)
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ddcosmo_gpu.h"

#define DDC_NLM_CAP ((DDC_MAX_LMAX + 1) * (DDC_MAX_LMAX + 2) / 2)

namespace ddc {

// Device buffer owned by a context (freed with it).
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    release();
    if (b == 0) b = 16;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

// Plan of the tensor-core contractions of the mixed-precision operators
// (ddc_tc.cu): tile widths, pipeline depths, the split images of the static
// operands, the TMA descriptor of the FP32 grid field and an error flag in
// mapped host memory that a kernel sets when one of its bounded waits runs out.
struct TcPlan {
  bool on = false;
  bool tuned = false;        // tile widths measured for tune_key's shape
  long long tune_key = 0;
  int tuned_bn_proj = 0, tuned_bn_xi = 0;
  bool xi_split = false, tuned_xi_split = false;  // expansion: one grid tile per CTA
  float ms_proj = 0.f, ms_xi = 0.f;  // measured launch times of the chosen widths
  int nsph = 0, nylm = 0, ngrid = 0, ldp = 0;
  int kc_proj = 0, bn_proj = 0, ns_proj = 0, smem_proj = 0;
  int mt_xi = 0, kc_xi = 0, bn_xi = 0, ns_xi = 0, smem_xi = 0;
  DBuf img_proj, img_xi;
  alignas(64) CUtensorMap tm_pot;
  float* pot_f = nullptr;
  int* err_h = nullptr;
  int* err_d = nullptr;
};

// Constants of the spherical-harmonic recurrences, indexed by (l, m >= 0)
// packed as l*(l+1)/2 + m.  Passed by value to the kernels (parameter space
// is a broadcast constant bank, so per-(l,m) reads are free).
struct YlmTables {
  double facl[DDC_MAX_LMAX + 1];  // (2l+1)/(4pi): D^-1 block (ddcosmo.f90:233)
  double facs[DDC_NLM_CAP];       // Y_lm normalisation incl. odd-m sign (:236-242)
  double K[DDC_NLM_CAP];          // facs / facl
  double A[DDC_NLM_CAP];          // (2l-1)/(l-m): Legendre recurrence
  double B[DDC_NLM_CAP];          // (l+m-1)/(l-m)
  float Kf[DDC_NLM_CAP], Af[DDC_NLM_CAP], Bf[DDC_NLM_CAP];  // FP32 copies (mixed path)
  // normalised recurrence of the fused L / L* kernel: Pt_l^m = gam_lm Q_l^m with
  // Q_m = Pt_m^m, Q_{m+1} = c t Q_m, Q_l = c t Q_{l-1} - beta_lm t^2 Q_{l-2};
  // Kg = K * gam folds the scale into the contractions
  double Bn[DDC_NLM_CAP], Kg[DDC_NLM_CAP];
  float Bnf[DDC_NLM_CAP];
  double eta;
  int lmax, nylm, ngrid;
};

// Device geometry handed to every kernel.
// Spheres a batched sweep may skip: those of molecules whose systems have
// all stopped (their operator outputs are not read again).  mol == null:
// every sphere is computed.
struct SweepMask {
  const int* mol;  // [nsph] molecule of each sphere
  const int* st0;  // [nmol] Jacobi/DIIS status of the first system (0: running)
  const int* st1;  // [nmol] status of the second system, or null
};

#ifdef __CUDACC__
// True for a sphere of a batched molecule whose systems have all stopped.
__device__ __forceinline__ bool sweep_skip(const SweepMask& m, int sph) {
  if (!m.mol) return false;
  const int k = m.mol[sph];
  return m.st0[k] != 0 && (!m.st1 || m.st1[k] != 0);
}
// True for every thread of the block when the spheres [i0, i0 + w) are all
// skipped (a block barrier: call it from every thread, w <= blockDim.x)
__device__ __forceinline__ bool sweep_skip_tile(const SweepMask& m, int i0, int w, int nsph) {
  if (!m.mol) return false;
  const int i = i0 + (int)threadIdx.x;
  return __syncthreads_and((int)threadIdx.x >= w || i >= nsph || sweep_skip(m, i)) != 0;
}
#endif

struct DevGeo {
  int nsph, ngrid, nylm, ncav, npair;
  int maxnb;  // largest neighbour count of a sphere
  // FP32 geometry of each gather-list triple (mixed path; null if absent):
  // (t cos theta, t^2, t sin theta, W) and (cos phi, sin phi)
  const float4* tgeo4;
  const float2* tgeo2;
  const double4* tgeo4d;  // the same in FP64 (FP64 path)
  const double2* tgeo2d;
  long long ntri;
  const double4* sph;
  const double4* grid;
  const float4* gridf;  // FP32 copy of grid (mixed path)
  const double* basis;
  const double* bw;
  const double* fi;
  const double* ui;
  const double* zi;
  const int* inl;
  const int* nl;
  const int* rev;
  const int* pn_ptr;
  const uint16_t* pn;
  const uint8_t* pn_pair;  // local index (within the sphere's CSR range) of each triple's pair
  const int* ls_ptr;
  const int2* ls;
  const int* lsstart;  // per CSR entry (j,i): start of that pair's block in i's gather list
  const uint8_t* ntri_pt;
  const int* cavoff;
  const int* cavidx;
  const int* cavpt;
  const double* ccav;
  SweepMask act;
};

// Stages timed with CUDA events when ddc_params.timing = 1.
enum Stage {
  ST_INIT = 0, ST_COULOMB, ST_RHS, ST_LX_POT, ST_PROJ, ST_XI, ST_LSTARX, ST_JACOBI,
  ST_COMBINE, ST_REDUCE, ST_UCHI, ST_FORCES, ST_ZETA, ST_EFIELD, ST_CONTRACT, ST_LXS,
  ST_GATHER, ST_N
};

// History of DIIS vectors for the fused Jacobi step / extrapolation.
constexpr int kMaxHist = 32;
// elements per chunk of the batched Jacobi/DIIS kernels
constexpr int kBatchChunk = 2048;
// The vectors are FP64, or FP32 for the inner solves of the mixed path.
struct HistPtrs {
  const void* p[kMaxHist];
  double c[kMaxHist];
  int n;
};

// Per-molecule Jacobi/DIIS state of a batched solve (device arrays).
struct BatchState {
  int nmol, ndiis, max_iter;
  double tol;
  long long n_total;  // length of the concatenated vectors
  const int* off;     // [nmol+1] sphere offsets
  int* nmat;          // [nmol]
  int* slot;          // [nmol][ndiis] logical -> physical history slot
  double* B;          // [nmol][(ndiis+1)^2] column-major bordered Gram matrix
  int* status;        // [nmol]: 0 active, 1 converged, 2 max_iter, 3 non-finite
  int* iters;         // [nmol]
  int* restarts;      // [nmol]
  double* norm;       // [nmol] last increment norm
  void* hx;           // [ndiis][n_total], FP64 or (f32) FP32
  void* he;           // [ndiis][n_total]
  int f32;            // history vectors in FP32 (inner solves of the mixed refinement)
  const double* tolk; // [nmol] per-molecule tolerance, or null: tol
  const int* maxk;    // [nmol] per-molecule iteration budget, or null: max_iter
  // element chunks of the per-molecule kernels: chunk c holds up to
  // kBatchChunk consecutive elements of molecule cmol[c]
  int nchunk;
  const int* cmol;    // [nchunk]
  const int* cfirst;  // [nmol+1] first chunk of each molecule
  double* part;       // [nchunk][kMaxHist+1] per-chunk partial sums
  unsigned* cnt;      // [nmol] arrival counters, zero between kernels
  double* coef;       // [nmol][kMaxHist] extrapolation coefficients
  int* ext;           // [nmol] terms of the extrapolation; negative after a singular solve
};

// ---------------------------------------------------------------------------
// Kernel launchers (ddc_kernels.cu).  All run on `st` and return the CUDA
// error of the launch.  `launches` is incremented per kernel launched.
// ---------------------------------------------------------------------------
struct Launch {
  cudaStream_t st;
  long long* launches;
};

// init
cudaError_t launch_basis(Launch L, const YlmTables& tb, const double4* grid, double* basis,
                         double* bw);
// mrange: per sphere, the index range of its molecule (nullptr: one molecule)
cudaError_t launch_csr_count(Launch L, int nsph, const double4* sph, int* cnt,
                             const int2* mrange);
cudaError_t launch_csr_fill(Launch L, int nsph, const double4* sph, const int* inl, int* nl,
                            const int2* mrange);
cudaError_t launch_csr_rev(Launch L, int nsph, const int* inl, const int* nl, int* rev);
// gord: the grid points in patch order (the threads of a warp take 32
// consecutive entries of one sphere)
cudaError_t launch_fiui(Launch L, const YlmTables& tb, int nsph, const double4* sph,
                        const double4* grid, const int* gord, const int* inl, const int* nl,
                        double* fi, double* ui, double* zi, uint8_t* ntri);
cudaError_t launch_cav_count(Launch L, int nsph, int ngrid, const double* ui, int* cnt);
cudaError_t launch_cav_fill(Launch L, int nsph, int ngrid, const double* ui, const double4* sph,
                            const double4* grid, const int* cavoff, int* cavidx, int* cavpt,
                            double* ccav);
cudaError_t launch_pair_count(Launch L, int nsph, int npair, int ngrid, const double4* sph,
                              const double4* grid, const int* inl, const int* nl, int* cnt,
                              unsigned* bits);  // bits: [npair][ceil(ngrid / 32)] words
cudaError_t launch_pair_fill(Launch L, int nsph, int npair, int ngrid, const double4* sph,
                             const double4* grid, const int* inl, const int* nl,
                             const unsigned* bits, const int* pn_ptr, uint16_t* pn,
                             uint8_t* pn_pair);
cudaError_t launch_ls_count(Launch L, int nsph, const int* inl, const int* rev, const int* pn_ptr,
                            int* cnt);
cudaError_t launch_ls_fill(Launch L, int nsph, const int* inl, const int* nl, const int* rev,
                           const int* pn_ptr, const uint16_t* pn, const int* ls_ptr, int2* ls,
                           int* lsstart);
// exclusive scan of n ints (out[n] = total); temp is device scratch of temp_bytes
cudaError_t scan_exclusive(Launch L, const int* in, int* out, int n, void* temp,
                           size_t temp_bytes);
size_t scan_temp_bytes(int n);
// *out = sum of cnt[0..n) in 64 bits (out: device memory, overwritten)
cudaError_t launch_sum_counts(Launch L, const int* cnt, int n, unsigned long long* out);

// operators
// xk: scratch of N*(lmax+1)(lmax+2)/2 double2 (K-scaled X in pair layout)
cudaError_t launch_lstarx_acc(Launch L, const YlmTables& tb, const DevGeo& g, const double* xi,
                              double* y);
// FP32 operator variants (mixed precision): pot/xi in FP32, y in FP64
// fused L / L*: val (one lx value per triple, gather-list order) and y = L* rows
cudaError_t launch_lxs(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                       const double* xi, void* xk, double* val, double* y);
// the lx part of the fused pass alone: one value per triple (gather-list
// order) for k_lx_gather; chi_only: weight chi(t) instead of chi(t)/f_a(n)
// (the u_chi sum of the forces)
cudaError_t launch_lx_vals(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                           void* xk, double* val, bool chi_only);
cudaError_t launch_lx_vals_f32(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                               void* xk, float* val);
cudaError_t launch_lxs_geo(Launch L, const YlmTables& tb, const DevGeo& g, float4* tg4,
                           float2* tg2);
cudaError_t launch_lxs_geo_f64(Launch L, const YlmTables& tb, const DevGeo& g, double4* tg4,
                               double2* tg2);
cudaError_t launch_lxs_f32(Launch L, const YlmTables& tb, const DevGeo& g, const double* X,
                           const float* xi, void* xk, float* val, double* y);
cudaError_t launch_lx_gather(Launch L, const DevGeo& g, const double* val, double* pot);
// FP32 field rows are ldp >= ngrid floats apart (the tensor-core projection
// reads them with TMA, which wants 16-byte row strides)
cudaError_t launch_lx_gather_f32(Launch L, const DevGeo& g, const float* val, float* pot,
                                 int ldp);
cudaError_t launch_lstarx_acc_f32(Launch L, const YlmTables& tb, const DevGeo& g,
                                  const float* xi, double* y);
cudaError_t launch_to_float(Launch L, long long n, const double* x, float* y);
// r = rhs - y - x/facl ; d = facl*r (Jacobi increment at x), partial H-norm of d
cudaError_t launch_residual(Launch L, const YlmTables& tb, long long n, const double* rhs,
                            const double* y, const double* x, double* r, double* d,
                            double* partials, int nblk);
cudaError_t launch_axpy(Launch L, long long n, double a, const double* x, double* y);
// dst[c*rows + r] = src[r*cols + c] (FP64)
cudaError_t launch_transpose(Launch L, int rows, int cols, const double* src, double* dst);
// C[n*ldc + m] = alpha * sum_k A[k*lda + m] B[n*ldb + k] (FP64, pipelined);
// with act.mol set the N columns are spheres and tiles of skipped spheres
// are left alone
cudaError_t launch_dgemm_nn(Launch L, int M, int N, int K, double alpha, const double* A,
                            int lda, const double* B, int ldb, double* C, int ldc,
                            const SweepMask& act = SweepMask{});
// FP32 SIMT projection / expansion (mixed path, more than 128 harmonics)
cudaError_t launch_proj_f32_simt(Launch L, int nylm, int nsph, int ngrid, float alpha,
                                 const float* bw_f, const float* pot, int ldp, double* y);
cudaError_t launch_xi_f32_simt(Launch L, int nylm, int nsph, int ngrid, const float* basis_f,
                               const double* s, float* xi);
cudaError_t launch_wghpot(Launch L, const DevGeo& g, const double* phi, double* gbuf);
cudaError_t launch_ldm1x(Launch L, const YlmTables& tb, long long n, const double* x, double* y);
cudaError_t launch_scale(Launch L, long long n, double a, const double* x, double* y);
cudaError_t launch_guess(Launch L, const YlmTables& tb, long long n, const double* rhs,
                         double* x, int mode);

// tensor-core contractions of the mixed-precision operators (ddc_tc.cu):
// projection y = alpha * bw pot (FP64 out) and expansion xi = basis^T s (FP32
// out), split-TF32 on tcgen05 for nylm <= 128
bool tc_supported(int nylm);
cudaError_t tc_plan(Launch L, TcPlan& p, const double* basis, const double* bw, int nsph,
                    int nylm, int ngrid, float* pot_f, int ldp);
// pick the tile widths of both kernels by timing the candidates (y, xi are
// scratch; s is zeroed)
cudaError_t tc_autotune(Launch L, TcPlan& p, const double* s, double* y, float* xi);
cudaError_t launch_proj_tc(Launch L, const TcPlan& p, double alpha, double* y,
                           const SweepMask& act = SweepMask{});
cudaError_t launch_xi_tc(Launch L, const TcPlan& p, const double* s, float* xi,
                         const SweepMask& act = SweepMask{});
void tc_release(TcPlan& p);

// learned initial guess (ddc_guess.cu)
int guess_nfeat(const ddc_guess* m);
int guess_nout(const ddc_guess* m);
int guess_lmax(const ddc_guess* m);
// raw per-sphere features [nsph][nin]: g (nylm), psi(00), radius, 16-bin
// histogram of the distances to the other centres of the sphere's molecule
cudaError_t launch_guess_features(Launch L, int nsph, int nylm, int nin, const double* g,
                                  const double* psi, const double4* sph, const int2* mrange,
                                  float* feat);
// training targets [nsph][nout]: X - facl g and S - facl psi
cudaError_t launch_guess_targets(Launch L, const YlmTables& tb, int nsph, int nout,
                                 const double* g, const double* psi, const double* X,
                                 const double* S, float* t);
// x = facl g + model correction, s = facl psi + model correction
cudaError_t guess_infer(Launch L, ddc_guess* m, const YlmTables& tb, int nsph, const float* feat,
                        const double* g, const double* psi, double* x, double* s);

// solver
// xnew = facl*(rhs - y); e = xnew - x; dots e.h_k (k < hist.n) and e.e.
// xnew, e and the history are FP32 when f32 (mixed-path inner solves), else FP64.
// The block partials go to partials; the last block sums them into out[0..hist.n]
// (counter: a zeroed device word, left zeroed).
cudaError_t launch_jacobi_step(Launch L, const YlmTables& tb, long long n, const double* rhs,
                               const double* y, const double* x, void* xnew, void* e,
                               const HistPtrs& hist, double* partials, int nblk, bool f32,
                               int* nblk_used,  // blocks launched (<= nblk): partial rows
                               unsigned* counter, double* out);
// xout = sum c_k p_k (or xjac if hist.n == 0); sum_l 1/(l+1) (xout-x)^2 into
// out[0] (through partials and counter as above); x = xout
cudaError_t launch_diis_combine(Launch L, const YlmTables& tb, long long n, const HistPtrs& hist,
                                const void* xjac, double* x, double* partials, int nblk,
                                bool f32, unsigned* counter, double* out);
cudaError_t launch_hnorm_partial(Launch L, const YlmTables& tb, long long n, const double* x,
                                 double* partials, int nblk);
cudaError_t launch_dot_partial(Launch L, long long n, const double* a, const double* b,
                               double* partials, int nblk);
// out[k] = sum_b partials[b*stride + k], k < nvals, fixed order; stride is
// the row length the producing kernel stores (block_sum_store's NV)
cudaError_t launch_reduce_partials(Launch L, const double* partials, int nblk, int nvals,
                                   int stride, double* out);
int reduce_blocks();

// electrostatics
// near / far split of the solute potential (and field) at the cavity points:
// charges farther than kFarRho * r_i from a sphere enter through a local
// expansion of degree kFarDegree about its centre, the others directly; used
// from kFarMinSpheres spheres on (below, the direct sums are cheaper)
constexpr int kFarDegree = 10;
constexpr double kFarRho = 8.0;
constexpr int kFarMinSpheres = 4096;
// BT[lm][n] = Y_lm(s_n), DT[k][lm][n] = grad_k R_lm(s_n) for the degree of tbP
cudaError_t launch_far_tables(Launch L, const YlmTables& tbP, const double4* grid, int ngrid,
                              double* BT, double* DT);
struct ZGroups;  // cell groups of one molecule (below)
// phi (and ef, if not null) at the cavity points; A: scratch [nsph][nylm(tbP)];
// zg (null for a batch): the near charges are searched in the candidate groups
cudaError_t launch_far_pot_field(Launch L, const YlmTables& tbP, int nsph, int ngrid,
                                 const double4* sph, const double* q, const int2* mrange,
                                 double rho, const int* cavoff, const int* cavpt,
                                 const double* ccav, const double* BT, const double* DT,
                                 double* A, double* phi, double* ef, const ZGroups* zg);
// Field of the cavity charges zeta at the nuclei in the mixed-precision
// energy+force flow (force-only, FP32 pair arithmetic): from
// kZetaMinSpheres spheres on, the spheres are grouped by the cells of a
// uniform grid (side >= kZetaCell bohr, Morton order), and a group farther
// than kZetaRho group radii from a nucleus acts through its multipole
// expansion of degree kZetaDegree; nearer groups are summed directly
constexpr int kZetaDegree = 16;
constexpr double kZetaRho = 3.0;
constexpr double kZetaCell = 12.0;
constexpr int kZetaMinSpheres = 4096;
// Cell groups of one molecule of kZetaMinSpheres spheres or more: the
// candidates of the neighbour list, of the near lists of the cavity far
// field and the source groups of the field of zeta
struct ZGroups {
  int ngroup = 0;
  int* cellid = nullptr;   // [nsph] scratch
  int* gsph = nullptr;     // [nsph] spheres in group order
  int* gstart = nullptr;   // [nsph+1] group g owns gsph[gstart[g] .. gstart[g+1])
  double4* gcen = nullptr; // [nsph] centroid and radius of each group
  int* gnpt = nullptr;     // [nsph+1] cavity points per group
  int* gptr = nullptr;     // [nsph+1] their exclusive scan
};
size_t zgroups_scan_bytes(int nsph);
// the cell groups of one molecule: members, centroids and radii (one host
// read of the group count); used by the neighbour list, the near lists of
// the cavity far field and the field of zeta
cudaError_t launch_zgroups_cells(Launch L, int nsph, const double4* sph, ZGroups& zg,
                                 int* dcount, int* hcount);
// per-group cavity-point counts and offsets (gnpt, gptr) for the field of zeta
cudaError_t launch_zgroups_points(Launch L, const int* cavoff, ZGroups& zg, void* scan_tmp,
                                  size_t scan_bytes);
// neighbour list of one molecule from its cell groups (same lists as
// launch_csr_count / launch_csr_fill)
cudaError_t launch_csr_count_cells(Launch L, int nsph, const double4* sph, const ZGroups& zg,
                                   int* cnt);
cudaError_t launch_csr_fill_cells(Launch L, int nsph, const double4* sph, const ZGroups& zg,
                                  const int* inl, int* nl);
int zgroups_nchunk(const ZGroups& zg);
size_t zgroups_moment_count(const ZGroups& zg);
// ef(3, nsph) from zeta(ncav); zpk[ncav], M[moment count], scratch
// [nchunk][nsph][3]
cudaError_t launch_zeta_field_far(Launch L, int nsph, const double4* sph, const int* cavoff,
                                  const double* ccav, const double* zeta, const ZGroups& zg,
                                  float4* zpk, float2* M, double* scratch, double* ef);
// trange: per target, the source index range it sums over (nullptr: all)
// launch_coulomb_pot plus the field of the same sources at the targets, ef (3, ntrg)
cudaError_t launch_coulomb_pot_field(Launch L, int nsrc, const double* q, const double* sx,
                                     const double* sy, const double* sz, int ntrg,
                                     const double* ctrg, double* phi, double* ef,
                                     const int2* trange);
cudaError_t launch_coulomb_pot(Launch L, int nsrc, const double* q, const double* sx,
                               const double* sy, const double* sz, int ntrg, const double* ctrg,
                               double* phi, const int2* trange);
cudaError_t launch_psi(Launch L, int n, int nylm, const double* q, double* psi);
// field of sources (q at csrc(3,nsrc)) at targets ctrg(3,ntrg); partial sums
// over `nchunk` source chunks go to scratch[nchunk][ntrg][3]
cudaError_t launch_efield(Launch L, int nsrc, const double* q, const double* csrc, int ntrg,
                          const double* ctrg, double* ef, double* scratch, int nchunk,
                          const int2* trange);
int efield_chunks(int nsrc, int ntrg);
// load k_efield / k_efield_reduce on the current device (one-time set-up)
cudaError_t preload_efield();
int efield_chunks_f32(int nsrc, int ntrg);
// FP32 pair arithmetic, FP64 accumulation (mixed-precision force terms)
cudaError_t launch_efield_f32(Launch L, int nsrc, const double* q, const double* csrc, int ntrg,
                              const double* ctrg, double* ef, double* scratch, int nchunk,
                              const int2* trange);

// forces
// fxa (3,N), fda (3,T) and fv (4 (lmax+1)(lmax+2)/2 pairs per sphere) are
// scratch of the force kernels
cudaError_t launch_forces(Launch L, const YlmTables& tb, const DevGeo& g, const double* sigma,
                          const double* s_xi, const double* u_chi, const double* phi,
                          double fep, double* fx, double* fxa, double* fda, double2* fv);
cudaError_t launch_mkxi(Launch L, const YlmTables& tb, const DevGeo& g, const double* xi_grid,
                        double scale, double* out);
cudaError_t launch_zeta_efld_contract(Launch L, const DevGeo& g, const double* zeta,
                                      const double* ef, double* fx);
cudaError_t launch_charge_efld_contract(Launch L, int n, const double* q, const double* ef,
                                        double* fx);
// batched solves
cudaError_t launch_batch_diis(Launch L, const YlmTables& tb, const BatchState& bs,
                              const double* rhs, const double* y, double* x);
// Mixed refinement of a batch, per molecule with run[k] == 0: r = rhs - y -
// x/facl, d = facl r (the FP64 Jacobi increment at x), e = d, and the
// increment's H-norm into norm[k] (chunk map and partials of bs).
cudaError_t launch_batch_residual(Launch L, const YlmTables& tb, const BatchState& bs,
                                  const int* run, const double* rhs, const double* y,
                                  const double* x, double* r, double* d, double* e, double* norm);
// x += e over the molecules with upd[k] != 0
cudaError_t launch_batch_update(Launch L, const BatchState& bs, int nylm, const int* upd,
                                const double* e, double* x);
cudaError_t launch_batch_dot(Launch L, int nmol, const int* off, int nylm, const double* a,
                             const double* b, double scale, double* out);
cudaError_t launch_batch_ranges(Launch L, int nsph, int ngrid, int ncav, const int2* mrange,
                                const int* cavpt, const int* cavoff, int2* tr_cav, int2* tr_nuc);

// FP64 FMA throughput probe: each thread runs `iters` x 8 independent FMA chains
cudaError_t launch_fp64_probe(Launch L, int blocks, int iters, double* out);
cudaError_t launch_fp32_probe(Launch L, int blocks, int iters, float* out);

cudaError_t launch_csph_pack(Launch L, int n, const double4* sph, double* csph, double* sx,
                             double* sy, double* sz);

}  // namespace ddc
