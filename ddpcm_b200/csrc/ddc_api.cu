// ddc_api.cu -- host side of the B200 ddCOSMO library: the C ABI of
// include/ddcosmo_gpu.h, the module state (context), the ddinit pipeline and
// the Jacobi/DIIS driver.  All device work runs on the context's stream.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>


#include "ddc_internal.h"
#include "lebedev_orbits.inc"

using namespace ddc;

namespace {

// ---------------------------------------------------------------------------
// device buffer
// ---------------------------------------------------------------------------
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// ---------------------------------------------------------------------------
// Lebedev grid (llgrid, llgnew.f:5-91).  Each orbit record {code, a, b, v}
// expands to its Oh-symmetric points (gen_oh, llgnew.f:93-681): for every
// coordinate pattern ("shape") of the orbit, the signs of the non-zero
// coordinates are enumerated with the first non-zero coordinate varying
// fastest.  This reproduces the reference's point order, which fixes the
// order of the cavity points.
// ---------------------------------------------------------------------------
int snap_ngrid(int ngrid) {
  int best = 0, inear = 100000;
  for (int i = 0; i < LEB_NSIZES; i++) {
    int d = std::abs(leb_sizes[i] - ngrid);
    if (d < inear) {
      inear = d;
      best = i;
    }
  }
  return leb_sizes[best];
}

void expand_orbit(int code, double a, double b, double v, std::vector<double>& out) {
  // shapes: indices into {0, a, b, c}; 0 = zero coordinate
  static const int shapes1[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  static const int shapes2[3][3] = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
  static const int shapes3[1][3] = {{1, 1, 1}};
  static const int shapes4[3][3] = {{1, 1, 2}, {1, 2, 1}, {2, 1, 1}};
  static const int shapes5[6][3] = {{1, 2, 0}, {2, 1, 0}, {1, 0, 2},
                                    {2, 0, 1}, {0, 1, 2}, {0, 2, 1}};
  static const int shapes6[6][3] = {{1, 2, 3}, {1, 3, 2}, {2, 1, 3},
                                    {2, 3, 1}, {3, 1, 2}, {3, 2, 1}};
  const int(*shp)[3] = nullptr;
  int nshape = 0;
  double c = 0.0;
  switch (code) {
    case 1: a = 1.0; shp = shapes1; nshape = 3; break;
    case 2: a = std::sqrt(0.5); shp = shapes2; nshape = 3; break;
    case 3: a = std::sqrt(1.0 / 3.0); shp = shapes3; nshape = 1; break;
    case 4: b = std::sqrt(1.0 - 2.0 * a * a); shp = shapes4; nshape = 3; break;
    case 5: b = std::sqrt(1.0 - a * a); shp = shapes5; nshape = 6; break;
    case 6: c = std::sqrt(1.0 - a * a - b * b); shp = shapes6; nshape = 6; break;
    default: return;
  }
  const double val[4] = {0.0, a, b, c};
  for (int s = 0; s < nshape; s++) {
    int nz[3], nnz = 0;
    for (int k = 0; k < 3; k++)
      if (shp[s][k]) nz[nnz++] = k;
    for (int sg = 0; sg < (1 << nnz); sg++) {
      double p[3];
      for (int k = 0; k < 3; k++) p[k] = val[shp[s][k]];
      for (int q = 0; q < nnz; q++)
        if (sg & (1 << q)) p[nz[q]] = -p[nz[q]];
      out.push_back(p[0]);
      out.push_back(p[1]);
      out.push_back(p[2]);
      out.push_back(v);
    }
  }
}

bool lebedev(int ngrid, std::vector<double>& g4) {
  int gi = -1;
  for (int i = 0; i < LEB_NSIZES; i++)
    if (leb_sizes[i] == ngrid) gi = i;
  if (gi < 0) return false;
  g4.clear();
  for (int o = 0; o < leb_orbit_cnt[gi]; o++) {
    const leb_orbit_rec& r = leb_orbits[leb_orbit_off[gi] + o];
    expand_orbit(r.code, r.a, r.b, r.v, g4);
  }
  const double pi = 4.0 * std::atan(1.0);
  for (size_t i = 3; i < g4.size(); i += 4) g4[i] = g4[i] * 4.0 * pi;
  return (int)(g4.size() / 4) == ngrid;
}

}  // namespace

// ---------------------------------------------------------------------------
// context (the module state of ddcosmo.f90:87-127)
// ---------------------------------------------------------------------------
struct ddc_ctx {
  ddc_params prm{};
  YlmTables tb{};
  cudaStream_t st = nullptr;
  bool own_stream = true;
  long long launches = 0;
  // stage timers: event pairs recorded around stages, resolved at sync points
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
  double st_ms[ST_N] = {0};
  long long st_calls[ST_N] = {0};
  std::string err;
  bool ready = false;
  int nsph = 0, ncav = 0, nylm = 0, ngrid = 0, npair = 0;
  long long ntri = 0;
  std::vector<double> h_grid;  // x,y,z,w per point
  std::vector<int> h_gord;     // grid points in patch order (k_fiui)
  DBuf gord;
  // geometry
  DBuf sph, grid, basis, bw, fi, ui, zi, inl, nl, rev, pn_ptr, pn, pn_pair, ls_ptr, ls, ntri_pt;
  DBuf lsstart, fxa, fda, fvec, xk;
  DBuf pn_bits;  // per pair, which grid points lie inside the neighbour (ddinit scratch)
  // batched molecules: partition, per-target N-body ranges, per-molecule DIIS state
  int nmol = 1;
  bool batch_init = false;  // set while ddc_batch_energy_forces initialises
  bool capturing = false;   // stream capture in progress: no stage events
  std::vector<int> h_off;
  DBuf b_cmol, b_cfirst, b_part, b_cnt, b_coef, b_ext;  // chunked batched Jacobi/DIIS
  DBuf b_sphmol;        // molecule of each sphere (batched solves)
  DBuf b_tolk, b_maxk;  // per-molecule tolerance and budget of the inner solves
  DBuf b_run, b_upd, b_onorm;  // mixed refinement of a batch: outer status, update mask, norms
  SweepMask sweep{};    // set while the batched sweeps are captured
  DBuf d_off, mrange, tr_cav, tr_nuc, b_nmat, b_slot, b_B, b_status, b_iters, b_restarts, b_norm,
      b_out;
  const int2* mrange_ptr() const { return nmol > 1 ? mrange.as<int2>() : nullptr; }
  int maxnb = 0;
  DBuf cavoff, cavidx, cavpt, ccav, cnt, scan_tmp;
  DBuf csph, cx, cy, cz;  // csph(3,n) and SoA centres
  // work
  DBuf pot, xig, gbuf, rhs, x, y, xn, partials, red, hist_x, hist_e;
  DBuf rcount;  // arrival counter of the solver kernels' last-block sums (kept zero)
  DBuf phi, psi, sigma, s, q, fx, zeta, ef1, ef2, ef_scratch, uchi;
  DBuf in1, in2, in3, in4, out1;  // staging for host-pointer calls
  // mixed precision: FP32 grid/basis copies, FP32 grid fields, refinement vectors
  DBuf gridf, basis_f, bw_f, pot_f, xi_f, rres, dres, eres;
  // FP32 static geometry of the gather-list triples (mixed path)
  DBuf tgeo4, tgeo2;
  bool tgeo_on = false;
  // FP64 static geometry of the gather-list triples (FP64 path)
  DBuf tgeo4d, tgeo2d;
  bool tgeo64_on = false;
  // second solve set (direct and adjoint solved together) and the fused
  // operator's per-triple lx values
  DBuf y2, xn2, hist_x2, hist_e2, rres2, dres2, eres2, tval;
  // the two dense contractions of every operator application (projection
  // onto the harmonics, expansion to the grid): basisT[Y][G] is the basis
  // transposed for the FP64 expansion; tc plans the tensor-core kernels of
  // the mixed path, whose FP32 grid field pot_f has rows ldp_f floats apart
  DBuf basisT;
  TcPlan tc;
  int ldp_f = 0;
  // learned initial guess: the attached model, its feature rows, and flags
  // for the flows (rhs/psi/sigma/s of the last flow are valid; the initial
  // guesses are already in place)
  ddc_guess* gmodel = nullptr;
  DBuf gfeat;
  bool have_flow = false, guess_preset = false;
  // near / far split of the solute potential and field at the cavity:
  // tables of degree kFarDegree on the grid, the per-sphere expansions
  YlmTables tbP{};
  DBuf farBT, farDT, farA;
  bool far_on = false;
  // grouped multipole field of zeta at the nuclei (mixed energy+force flow)
  DBuf zg_cell, zg_sph, zg_start, zg_cen, zg_npt, zg_ptr, zg_cnt, zg_tmp, zg_M, zg_pk, zg_scr;
  ZGroups zg;
  bool zg_on = false;  // cell groups built for this molecule (single molecule, >= 4,096 spheres)
  bool zfar_on = false;
  // pinned landing buffer of the small device-to-host reads (reduced sums)
  double* hred = nullptr;
  // second stream of the force tail: the field of zeta at the nuclei runs
  // beside the force kernels (events: fork after zeta, join before its use)
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  unsigned int stage_mask = ~0u;  // stages timed when prm.timing is set

  Launch L() { return Launch{st, &launches}; }
  DevGeo geo() const {
    DevGeo g;
    g.nsph = nsph;
    g.ngrid = ngrid;
    g.nylm = nylm;
    g.ncav = ncav;
    g.npair = npair;
    g.ntri = ntri;
    g.sph = sph.as<double4>();
    g.grid = grid.as<double4>();
    g.gridf = gridf.as<float4>();
    g.basis = basis.as<double>();
    g.bw = bw.as<double>();
    g.fi = fi.as<double>();
    g.ui = ui.as<double>();
    g.zi = zi.as<double>();
    g.inl = inl.as<int>();
    g.nl = nl.as<int>();
    g.rev = rev.as<int>();
    g.pn_ptr = pn_ptr.as<int>();
    g.pn = pn.as<uint16_t>();
    g.pn_pair = pn_pair.as<uint8_t>();
    g.maxnb = maxnb;
    g.tgeo4 = tgeo_on ? tgeo4.as<float4>() : nullptr;
    g.tgeo2 = tgeo_on ? tgeo2.as<float2>() : nullptr;
    g.tgeo4d = tgeo64_on ? tgeo4d.as<double4>() : nullptr;
    g.tgeo2d = tgeo64_on ? tgeo2d.as<double2>() : nullptr;
    g.ls_ptr = ls_ptr.as<int>();
    g.ls = ls.as<int2>();
    g.lsstart = lsstart.as<int>();
    g.ntri_pt = ntri_pt.as<uint8_t>();
    g.cavoff = cavoff.as<int>();
    g.cavidx = cavidx.as<int>();
    g.cavpt = cavpt.as<int>();
    g.ccav = ccav.as<double>();
    g.act = sweep;
    return g;
  }
};

namespace {

int fail(ddc_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

// On failure the runtime's last-error state is cleared as well, so that a
// rejected launch configuration does not resurface in a later call.
#define CK(expr)                                                                          \
  do {                                                                                    \
    cudaError_t _e = (expr);                                                              \
    if (_e != cudaSuccess) {                                                              \
      cudaGetLastError();                                                                 \
      return fail(ctx, _e == cudaErrorMemoryAllocation ? DDC_ERR_NOMEM : DDC_ERR_CUDA,    \
                  std::string(#expr) + ": " + cudaGetErrorString(_e));                    \
    }                                                                                     \
  } while (0)

#define CKI(expr)                  \
  do {                             \
    int _r = (expr);               \
    if (_r != DDC_OK) return _r;   \
  } while (0)

// input array: device pointer as is, host array copied into staging
int stage_in(ddc_ctx* ctx, const double* p, size_t count, DBuf& buf, const double** out) {
  if (count == 0) {
    *out = p;
    return DDC_OK;
  }
  if (!p) return fail(ctx, DDC_ERR_PARAM, "null input array");
  if (ctx->prm.device_pointers) {
    *out = p;
    return DDC_OK;
  }
  CK(buf.ensure(count * sizeof(double)));
  CK(cudaMemcpyAsync(buf.p, p, count * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  *out = buf.as<double>();
  return DDC_OK;
}
// output: device pointer written directly; host array via a device buffer
int out_ptr(ddc_ctx* ctx, double* p, size_t count, DBuf& buf, double** dev) {
  if (ctx->prm.device_pointers && p) {
    *dev = p;
    return DDC_OK;
  }
  CK(buf.ensure((count ? count : 1) * sizeof(double)));
  *dev = buf.as<double>();
  return DDC_OK;
}
int finish_out(ddc_ctx* ctx, double* p, const double* dev, size_t count) {
  if (p && dev != p && count)
    CK(cudaMemcpyAsync(p, dev, count * sizeof(double),
                       ctx->prm.device_pointers ? cudaMemcpyDeviceToDevice
                                                : cudaMemcpyDeviceToHost,
                       ctx->st));
  return DDC_OK;
}
// Stage-timer events are turned into times in batches: resolving them at
// every synchronisation would put that host work between a solver step's
// reduction and its next launch.
void resolve_timers(ddc_ctx* ctx) {
  for (auto& pe : ctx->ev_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess) {
      ctx->st_ms[pe.first] += ms;
      ctx->st_calls[pe.first] += 1;
    }
    ctx->ev_pool.push_back(pe.second.first);
    ctx->ev_pool.push_back(pe.second.second);
  }
  ctx->ev_pending.clear();
}

int sync(ddc_ctx* ctx) {
  CK(cudaStreamSynchronize(ctx->st));
  if (ctx->tc.err_h && *ctx->tc.err_h) {
    const int code = *ctx->tc.err_h;
    *ctx->tc.err_h = 0;
    return fail(ctx, DDC_ERR_CUDA,
                "tensor-core contraction gave up waiting (code " + std::to_string(code) + ")");
  }
  if (ctx->ev_pending.size() >= 1024) resolve_timers(ctx);
  return DDC_OK;
}

// Times the enclosed launches on the context stream (when timing is on).
struct StageScope {
  ddc_ctx* c;
  int stage;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEvent_t take() {
    cudaEvent_t e = nullptr;
    if (!c->ev_pool.empty()) {
      e = c->ev_pool.back();
      c->ev_pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
      e = nullptr;
    }
    return e;
  }
  cudaStream_t on;
  StageScope(ddc_ctx* ctx, int s, cudaStream_t stream = nullptr)
      : c(ctx), stage(s), on(stream ? stream : ctx->st) {
    if (!c->prm.timing || c->capturing || !((c->stage_mask >> s) & 1u)) return;
    a = take();
    b = take();
    if (a && b) cudaEventRecord(a, on);
  }
  ~StageScope() {
    if (!a || !b) return;
    cudaEventRecord(b, on);
    c->ev_pending.push_back({stage, {a, b}});
  }
};

void build_tables_for(YlmTables& tb, int lmax, double eta, int ngrid) {
  memset(&tb, 0, sizeof(tb));
  const double pi = 4.0 * std::atan(1.0), sq2 = std::sqrt(2.0);
  std::vector<double> fact(std::max(2 * lmax + 1, 2));
  fact[0] = 1.0;
  fact[1] = 1.0;
  for (int i = 3; i <= 2 * lmax + 1; i++) fact[i - 1] = (double)(i - 1) * fact[i - 2];
  for (int l = 0; l <= lmax; l++) {
    double fl = (2.0 * (double)l + 1.0) / (4.0 * pi);
    double ffl = std::sqrt(fl);
    tb.facl[l] = fl;
    tb.facs[l * (l + 1) / 2] = ffl;
    for (int m = 1; m <= l; m++) {
      double fnorm = sq2 * ffl * std::sqrt(fact[l - m] / fact[l + m]);
      if (m % 2 == 1) fnorm = -fnorm;
      tb.facs[l * (l + 1) / 2 + m] = fnorm;
    }
    for (int m = 0; m <= l; m++) {
      int e = l * (l + 1) / 2 + m;
      tb.K[e] = tb.facs[e] / fl;
      if (l >= m + 2) {
        tb.A[e] = (2.0 * l - 1.0) / (double)(l - m);
        tb.B[e] = ((double)(l + m) - 1.0) / (double)(l - m);
      }
    }
  }
  for (int m = 0; m <= lmax; m++) {
    double gm2 = 1.0, gm1 = 1.0;  // gam_{l-2}, gam_{l-1}
    for (int l = m; l <= lmax; l++) {
      const int e = l * (l + 1) / 2 + m;
      double gam;
      if (l == m) {
        gam = 1.0;
      } else if (l == m + 1) {
        gam = 2.0 * m + 1.0;
      } else {
        gam = tb.A[e] * gm1;
        tb.Bn[e] = tb.B[e] * gm2 / gam;
      }
      tb.Kg[e] = tb.K[e] * gam;
      gm2 = gm1;
      gm1 = gam;
    }
  }
  for (int e = 0; e < DDC_NLM_CAP; e++) {
    tb.Kf[e] = (float)tb.K[e];
    tb.Af[e] = (float)tb.A[e];
    tb.Bf[e] = (float)tb.B[e];
    tb.Bnf[e] = (float)tb.Bn[e];
  }
  tb.eta = eta;
  tb.lmax = lmax;
  tb.nylm = (lmax + 1) * (lmax + 1);
  tb.ngrid = ngrid;
}
void build_tables(ddc_ctx* c) {
  build_tables_for(c->tb, c->prm.lmax, c->prm.eta, c->ngrid);
  // the degree of the far-field expansions of the solute potential
  build_tables_for(c->tbP, kFarDegree, c->prm.eta, c->ngrid);
}

// deterministic reduction of `nvals` partial columns into red[0..nvals-1], copied to host.
// stride: the partial row length of the producing kernel (kMaxHist + 1 for the
// Jacobi step's Gram row, whatever its current length; 1 for single sums).
// nblk: the producing kernel's block count (partial rows).
int reduce_to_host(ddc_ctx* ctx, int nvals, double* host, int stride = 1, int nblk = 0) {
  if (nvals > kMaxHist + 1 || !ctx->hred)
    return fail(ctx, DDC_ERR_STATE, "reduction read beyond the pinned buffer");
  {
    StageScope sc(ctx, ST_REDUCE);
    CK(launch_reduce_partials(ctx->L(), ctx->partials.as<double>(),
                              nblk > 0 ? nblk : reduce_blocks(), nvals, stride,
                              ctx->red.as<double>()));
  }
  CK(cudaMemcpyAsync(ctx->hred, ctx->red.p, sizeof(double) * nvals, cudaMemcpyDeviceToHost,
                     ctx->st));
  CKI(sync(ctx));
  memcpy(host, ctx->hred, sizeof(double) * nvals);
  return DDC_OK;
}

// The per-item counts that are about to be scanned into 32-bit offsets must
// total less than 2^31: summed in 64 bits on the device first.
int check_count_total(ddc_ctx* ctx, const int* cnt, int n, const char* what) {
  if (n <= 0) return DDC_OK;
  unsigned long long* d = reinterpret_cast<unsigned long long*>(ctx->red.p);
  CK(launch_sum_counts(ctx->L(), cnt, n, d));
  unsigned long long total = 0;
  CK(cudaMemcpyAsync(&total, d, sizeof(total), cudaMemcpyDeviceToHost, ctx->st));
  CKI(sync(ctx));
  if (total >= (unsigned long long)INT_MAX)
    return fail(ctx, DDC_ERR_UNSUPPORTED,
                std::string("more than 2^31 - 1 ") + what + " (" + std::to_string(total) + ")");
  return DDC_OK;
}

// ---------------------------------------------------------------------------
// ddinit (ddcosmo.f90:159-483) on device buffers
// ---------------------------------------------------------------------------
int do_init(ddc_ctx* ctx, int n, const std::vector<double4>* hsph, const double4* dsph) {
  ctx->ready = false;
  ctx->tgeo_on = false;
  ctx->tgeo64_on = false;
  ctx->nsph = n;
  ctx->nylm = (ctx->prm.lmax + 1) * (ctx->prm.lmax + 1);
  ctx->ngrid = snap_ngrid(ctx->prm.ngrid);
  build_tables(ctx);
  if (!lebedev(ctx->ngrid, ctx->h_grid)) return fail(ctx, DDC_ERR_PARAM, "bad Lebedev size");
  const int N = n, G = ctx->ngrid, NY = ctx->nylm;
  const long long NP = (long long)N * G;
  // grid fields, cavity and triple lists are indexed with 32-bit integers
  if (NP >= (long long)INT_MAX)
    return fail(ctx, DDC_ERR_UNSUPPORTED, "nsph * ngrid exceeds 2^31 - 1 grid points");
  // two rows (the direct and adjoint solves' reductions); also the count checks' scratch
  CK(ctx->red.ensure(sizeof(double) * 2 * (kMaxHist + 1)));
  auto L = ctx->L();
  CK(ctx->sph.ensure(sizeof(double4) * std::max(N, 1)));
  if (hsph)
    CK(cudaMemcpyAsync(ctx->sph.p, hsph->data(), sizeof(double4) * N, cudaMemcpyHostToDevice,
                       ctx->st));
  else if (dsph != ctx->sph.as<double4>())
    CK(cudaMemcpyAsync(ctx->sph.p, dsph, sizeof(double4) * N, cudaMemcpyDeviceToDevice, ctx->st));
  CK(ctx->grid.ensure(sizeof(double4) * G));
  CK(cudaMemcpyAsync(ctx->grid.p, ctx->h_grid.data(), sizeof(double4) * G, cudaMemcpyHostToDevice,
                     ctx->st));
  {
    // grid points in Morton order of their directions: 32 consecutive
    // entries form a compact patch of the sphere, so that the warps of the
    // per-point neighbour loop (k_fiui) skip whole neighbours whose cap
    // misses their patch
    std::vector<std::pair<uint64_t, int>> key(G);
    for (int k = 0; k < G; k++) {
      uint64_t m = 0;
      uint32_t c[3];
      for (int d = 0; d < 3; d++)
        c[d] = (uint32_t)std::min(1023.0, std::floor((ctx->h_grid[4 * k + d] + 1.0) * 511.75));
      for (int b = 9; b >= 0; b--)
        for (int d = 0; d < 3; d++) m = (m << 1) | ((c[d] >> b) & 1u);
      key[k] = {m, k};
    }
    std::sort(key.begin(), key.end());
    ctx->h_gord.resize(G);
    for (int k = 0; k < G; k++) ctx->h_gord[k] = key[k].second;
    CK(ctx->gord.ensure(sizeof(int) * G));
    CK(cudaMemcpyAsync(ctx->gord.p, ctx->h_gord.data(), sizeof(int) * G, cudaMemcpyHostToDevice,
                       ctx->st));
  }
  CK(ctx->basis.ensure(sizeof(double) * G * NY));
  CK(ctx->bw.ensure(sizeof(double) * G * NY));
  CK(launch_basis(L, ctx->tb, ctx->grid.as<double4>(), ctx->basis.as<double>(),
                  ctx->bw.as<double>()));
  // cell groups of one large molecule: candidates for the neighbour list,
  // the near lists of the cavity far field and the groups of the field of
  // zeta (DDC_CELLS_OFF=1 keeps the all-pairs scans: a diagnostic switch)
  {
    const char* coff = std::getenv("DDC_CELLS_OFF");
    ctx->zg_on = ctx->nmol <= 1 && N >= kZetaMinSpheres && !(coff && coff[0] == '1');
    if (ctx->zg_on) {
      CK(ctx->zg_cell.ensure(sizeof(int) * N));
      CK(ctx->zg_sph.ensure(sizeof(int) * N));
      CK(ctx->zg_start.ensure(sizeof(int) * (N + 1)));
      CK(ctx->zg_cen.ensure(sizeof(double4) * N));
      CK(ctx->zg_cnt.ensure(sizeof(int)));
      ZGroups& z = ctx->zg;
      z.cellid = ctx->zg_cell.as<int>();
      z.gsph = ctx->zg_sph.as<int>();
      z.gstart = ctx->zg_start.as<int>();
      z.gcen = ctx->zg_cen.as<double4>();
      z.gnpt = nullptr;
      z.gptr = nullptr;
      if (!ctx->hred) CK(cudaMallocHost(&ctx->hred, sizeof(double) * 2 * (kMaxHist + 1)));
      CK(launch_zgroups_cells(L, N, ctx->sph.as<double4>(), z, ctx->zg_cnt.as<int>(),
                              reinterpret_cast<int*>(ctx->hred)));
    }
  }
  // neighbour list
  size_t scan_n = (size_t)std::max<long long>(N, 1);
  CK(ctx->cnt.ensure(sizeof(int) * (scan_n + 1)));
  CK(ctx->inl.ensure(sizeof(int) * (N + 1)));
  CK(cudaMemsetAsync(ctx->cnt.p, 0, sizeof(int) * (N + 1), ctx->st));
  if (N > 0) {
    if (ctx->zg_on)
      CK(launch_csr_count_cells(L, N, ctx->sph.as<double4>(), ctx->zg, ctx->cnt.as<int>()));
    else
      CK(launch_csr_count(L, N, ctx->sph.as<double4>(), ctx->cnt.as<int>(), ctx->mrange_ptr()));
  }
  size_t tb_bytes = scan_temp_bytes(N);
  CK(ctx->scan_tmp.ensure(tb_bytes));
  CKI(check_count_total(ctx, ctx->cnt.as<int>(), N, "neighbour pairs"));
  CK(scan_exclusive(L, ctx->cnt.as<int>(), ctx->inl.as<int>(), N, ctx->scan_tmp.p, tb_bytes));
  int npair = 0;
  CK(cudaMemcpyAsync(&npair, ctx->inl.as<int>() + N, sizeof(int), cudaMemcpyDeviceToHost,
                     ctx->st));
  CKI(sync(ctx));
  ctx->npair = npair;
  CK(ctx->nl.ensure(sizeof(int) * std::max(npair, 1)));
  CK(ctx->rev.ensure(sizeof(int) * std::max(npair, 1)));
  {
    std::vector<int> h_inl(N + 1);
    CK(cudaMemcpyAsync(h_inl.data(), ctx->inl.p, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost,
                       ctx->st));
    CKI(sync(ctx));
    int mx = 0;
    for (int i = 0; i < N; i++) mx = std::max(mx, h_inl[i + 1] - h_inl[i]);
    ctx->maxnb = mx;
    // the lx kernel indexes a sphere's neighbours with 8 bits (the reference
    // caps the list at nngmax = 100 per sphere on average, ddcosmo.f90:87)
    const size_t smem = 32 * (size_t)mx + 4 * (size_t)mx + 32 * (size_t)G;
    if (mx > 255 || smem > 200 * 1024)
      return fail(ctx, DDC_ERR_UNSUPPORTED, "a sphere has too many neighbours (" +
                                                std::to_string(mx) + ")");
  }
  if (N > 0) {
    if (ctx->zg_on)
      CK(launch_csr_fill_cells(L, N, ctx->sph.as<double4>(), ctx->zg, ctx->inl.as<int>(),
                               ctx->nl.as<int>()));
    else
      CK(launch_csr_fill(L, N, ctx->sph.as<double4>(), ctx->inl.as<int>(), ctx->nl.as<int>(),
                         ctx->mrange_ptr()));
    CK(launch_csr_rev(L, N, ctx->inl.as<int>(), ctx->nl.as<int>(), ctx->rev.as<int>()));
  }
  // fi, ui, zi
  CK(ctx->fi.ensure(sizeof(double) * std::max(NP, 1LL)));
  CK(ctx->ui.ensure(sizeof(double) * std::max(NP, 1LL)));
  CK(ctx->ntri_pt.ensure(std::max(NP, 1LL)));
  if (ctx->prm.igrad) CK(ctx->zi.ensure(sizeof(double) * 3 * std::max(NP, 1LL)));
  else ctx->zi.release();
  CK(launch_fiui(L, ctx->tb, N, ctx->sph.as<double4>(), ctx->grid.as<double4>(),
                 ctx->gord.as<int>(), ctx->inl.as<int>(), ctx->nl.as<int>(), ctx->fi.as<double>(),
                 ctx->ui.as<double>(),
                 ctx->prm.igrad ? ctx->zi.as<double>() : nullptr, ctx->ntri_pt.as<uint8_t>()));
  // cavity
  CK(ctx->cavoff.ensure(sizeof(int) * (N + 1)));
  CK(cudaMemsetAsync(ctx->cnt.p, 0, sizeof(int) * (N + 1), ctx->st));
  CK(launch_cav_count(L, N, G, ctx->ui.as<double>(), ctx->cnt.as<int>()));
  CK(scan_exclusive(L, ctx->cnt.as<int>(), ctx->cavoff.as<int>(), N, ctx->scan_tmp.p, tb_bytes));
  int ncav = 0;
  CK(cudaMemcpyAsync(&ncav, ctx->cavoff.as<int>() + N, sizeof(int), cudaMemcpyDeviceToHost,
                     ctx->st));
  CKI(sync(ctx));
  ctx->ncav = ncav;
  CK(ctx->cavidx.ensure(sizeof(int) * std::max(NP, 1LL)));
  CK(ctx->cavpt.ensure(sizeof(int) * std::max(ncav, 1)));
  CK(ctx->ccav.ensure(sizeof(double) * 3 * std::max(ncav, 1)));
  CK(launch_cav_fill(L, N, G, ctx->ui.as<double>(), ctx->sph.as<double4>(),
                     ctx->grid.as<double4>(), ctx->cavoff.as<int>(), ctx->cavidx.as<int>(),
                     ctx->cavpt.as<int>(), ctx->ccav.as<double>()));
  // pair-major triple lists
  size_t pscan = (size_t)std::max(npair, 1);
  CK(ctx->cnt.ensure(sizeof(int) * (std::max(scan_n, pscan) + 1)));
  CK(ctx->pn_ptr.ensure(sizeof(int) * (npair + 1)));
  CK(cudaMemsetAsync(ctx->cnt.p, 0, sizeof(int) * (npair + 1), ctx->st));
  CK(ctx->pn_bits.ensure(sizeof(unsigned) * std::max(npair, 1) * (size_t)((G + 31) / 32)));
  CK(launch_pair_count(L, N, npair, G, ctx->sph.as<double4>(), ctx->grid.as<double4>(),
                       ctx->inl.as<int>(), ctx->nl.as<int>(), ctx->cnt.as<int>(),
                       ctx->pn_bits.as<unsigned>()));
  CKI(check_count_total(ctx, ctx->cnt.as<int>(), npair, "(sphere, point, neighbour) triples"));
  size_t tb2 = scan_temp_bytes(npair);
  CK(ctx->scan_tmp.ensure(std::max(tb_bytes, tb2)));
  CK(scan_exclusive(L, ctx->cnt.as<int>(), ctx->pn_ptr.as<int>(), npair, ctx->scan_tmp.p,
                    ctx->scan_tmp.bytes));
  int ntri = 0;
  CK(cudaMemcpyAsync(&ntri, ctx->pn_ptr.as<int>() + npair, sizeof(int), cudaMemcpyDeviceToHost,
                     ctx->st));
  CKI(sync(ctx));
  ctx->ntri = ntri;
  CK(ctx->pn.ensure(sizeof(uint16_t) * std::max(ntri, 1)));
  CK(ctx->pn_pair.ensure(std::max(ntri, 1)));
  CK(launch_pair_fill(L, N, npair, G, ctx->sph.as<double4>(), ctx->grid.as<double4>(),
                      ctx->inl.as<int>(), ctx->nl.as<int>(), ctx->pn_bits.as<unsigned>(),
                      ctx->pn_ptr.as<int>(), ctx->pn.as<uint16_t>(), ctx->pn_pair.as<uint8_t>()));
  CK(ctx->ls_ptr.ensure(sizeof(int) * (N + 1)));
  CK(cudaMemsetAsync(ctx->cnt.p, 0, sizeof(int) * (N + 1), ctx->st));
  CK(launch_ls_count(L, N, ctx->inl.as<int>(), ctx->rev.as<int>(), ctx->pn_ptr.as<int>(),
                     ctx->cnt.as<int>()));
  CK(scan_exclusive(L, ctx->cnt.as<int>(), ctx->ls_ptr.as<int>(), N, ctx->scan_tmp.p,
                    ctx->scan_tmp.bytes));
  CK(ctx->ls.ensure(sizeof(int2) * std::max(ntri, 1)));
  CK(ctx->lsstart.ensure(sizeof(int) * std::max(npair, 1)));
  CK(launch_ls_fill(L, N, ctx->inl.as<int>(), ctx->nl.as<int>(), ctx->rev.as<int>(),
                    ctx->pn_ptr.as<int>(), ctx->pn.as<uint16_t>(), ctx->ls_ptr.as<int>(),
                    ctx->ls.as<int2>(), ctx->lsstart.as<int>()));
  // centres for the electrostatics
  CK(ctx->csph.ensure(sizeof(double) * 3 * std::max(N, 1)));
  CK(ctx->cx.ensure(sizeof(double) * std::max(N, 1)));
  CK(ctx->cy.ensure(sizeof(double) * std::max(N, 1)));
  CK(ctx->cz.ensure(sizeof(double) * std::max(N, 1)));
  CK(launch_csph_pack(L, N, ctx->sph.as<double4>(), ctx->csph.as<double>(), ctx->cx.as<double>(),
                      ctx->cy.as<double>(), ctx->cz.as<double>()));
  // solver work buffers
  const size_t nv = (size_t)N * NY;
  const int nd = std::max(ctx->prm.ndiis, 1);
  CK(ctx->pot.ensure(sizeof(double) * std::max(NP, 1LL)));
  CK(ctx->xk.ensure(sizeof(double) * 2 * std::max(N, 1) *
                    ((ctx->prm.lmax + 1) * (ctx->prm.lmax + 2) / 2)));
  CK(ctx->xig.ensure(sizeof(double) * std::max(NP, 1LL)));
  CK(ctx->uchi.ensure(sizeof(double) * std::max(NP, 1LL)));
  for (DBuf* b : {&ctx->rhs, &ctx->x, &ctx->y, &ctx->xn, &ctx->psi, &ctx->sigma, &ctx->s})
    CK(b->ensure(sizeof(double) * std::max(nv, (size_t)1)));
  CK(ctx->hist_x.ensure(sizeof(double) * std::max(nv, (size_t)1) * nd));
  CK(ctx->hist_e.ensure(sizeof(double) * std::max(nv, (size_t)1) * nd));
  CK(ctx->partials.ensure(sizeof(double) * reduce_blocks() * (kMaxHist + 1)));
  CK(ctx->red.ensure(sizeof(double) * 2 * (kMaxHist + 1)));
  if (!ctx->rcount.p) {
    CK(ctx->rcount.ensure(sizeof(unsigned)));
    CK(cudaMemsetAsync(ctx->rcount.p, 0, sizeof(unsigned), ctx->st));
  }
  // the basis transposed to [Y][G] for the FP64 expansion xi = basis^T s
  CK(ctx->basisT.ensure(sizeof(double) * G * NY));
  CK(launch_transpose(L, G, NY, ctx->basis.as<double>(), ctx->basisT.as<double>()));
  if (!ctx->hred) CK(cudaMallocHost(&ctx->hred, sizeof(double) * 2 * (kMaxHist + 1)));
  if (ctx->prm.igrad && !ctx->st2) {
    CK(cudaStreamCreateWithFlags(&ctx->st2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  }
  if (ctx->prm.precision == DDC_PREC_MIXED) {
    std::vector<float> gf(4 * (size_t)G);
    for (size_t k = 0; k < gf.size(); k++) gf[k] = (float)ctx->h_grid[k];
    CK(ctx->gridf.ensure(sizeof(float) * 4 * G));
    CK(cudaMemcpyAsync(ctx->gridf.p, gf.data(), sizeof(float) * 4 * G, cudaMemcpyHostToDevice,
                       ctx->st));
    // the two contractions run on the tensor cores (split TF32) up to 128
    // harmonics (lmax 10), else as FP32 SIMT GEMMs on FP32 copies of the basis
    // DDC_TC_OFF=1 in the environment selects the SIMT contractions (a
    // diagnostic switch: the tests compare the two paths' accuracy)
    const char* tc_off = std::getenv("DDC_TC_OFF");
    const bool tc = tc_supported(NY) && !(tc_off && tc_off[0] == '1');
    ctx->ldp_f = tc ? (G + 3) / 4 * 4 : G;
    CK(ctx->pot_f.ensure(sizeof(float) * std::max<long long>((long long)N * ctx->ldp_f, 1LL)));
    CK(ctx->xi_f.ensure(sizeof(float) * std::max(NP, 1LL)));
    if (tc) {
      CK(tc_plan(L, ctx->tc, ctx->basis.as<double>(), ctx->bw.as<double>(), N, NY, G,
                 ctx->pot_f.as<float>(), ctx->ldp_f));
      // tile widths by measurement (x and y are free work vectors here)
      CK(tc_autotune(L, ctx->tc, ctx->x.as<double>(), ctx->y.as<double>(),
                     ctx->xi_f.as<float>()));
    } else {
      ctx->tc.on = false;
      CK(ctx->basis_f.ensure(sizeof(float) * G * NY));
      CK(ctx->bw_f.ensure(sizeof(float) * G * NY));
      CK(launch_to_float(L, (long long)G * NY, ctx->basis.as<double>(), ctx->basis_f.as<float>()));
      CK(launch_to_float(L, (long long)G * NY, ctx->bw.as<double>(), ctx->bw_f.as<float>()));
    }
    for (DBuf* b : {&ctx->rres, &ctx->dres, &ctx->eres})
      CK(b->ensure(sizeof(double) * std::max(nv, (size_t)1)));
    // the FP32 fused pass reads each triple's static geometry instead of
    // recomputing it every iteration (24 bytes per triple)
    ctx->tgeo_on = false;
    CK(ctx->tgeo4.ensure(sizeof(float4) * std::max<long long>(ctx->ntri, 1)));
    CK(ctx->tgeo2.ensure(sizeof(float2) * std::max<long long>(ctx->ntri, 1)));
    CK(launch_lxs_geo(L, ctx->tb, ctx->geo(), ctx->tgeo4.as<float4>(), ctx->tgeo2.as<float2>()));
    ctx->tgeo_on = true;
  }
  if (ctx->prm.precision != DDC_PREC_MIXED && ctx->prm.pair_solves) {
    // the FP64 fused pass of the paired solves reads each triple's static
    // geometry (48 bytes per triple) instead of recomputing it
    CK(ctx->tgeo4d.ensure(sizeof(double4) * std::max<long long>(ctx->ntri, 1)));
    CK(ctx->tgeo2d.ensure(sizeof(double2) * std::max<long long>(ctx->ntri, 1)));
    CK(launch_lxs_geo_f64(L, ctx->tb, ctx->geo(), ctx->tgeo4d.as<double4>(),
                          ctx->tgeo2d.as<double2>()));
    ctx->tgeo64_on = true;
  }
  if (ctx->prm.igrad && ctx->prm.pair_solves) {
    for (DBuf* b : {&ctx->y2, &ctx->xn2})
      CK(b->ensure(sizeof(double) * std::max(nv, (size_t)1)));
    CK(ctx->hist_x2.ensure(sizeof(double) * std::max(nv, (size_t)1) * nd));
    CK(ctx->hist_e2.ensure(sizeof(double) * std::max(nv, (size_t)1) * nd));
    if (ctx->prm.precision == DDC_PREC_MIXED)
      for (DBuf* b : {&ctx->rres2, &ctx->dres2, &ctx->eres2})
        CK(b->ensure(sizeof(double) * std::max(nv, (size_t)1)));
  }
  // per-triple lx values of the fused passes (FP64 size: the mixed path also
  // takes FP64 steps in its refinement)
  CK(ctx->tval.ensure(sizeof(double) * std::max<long long>(ctx->ntri, 1)));
  // near / far split of the solute potential at the cavity for large systems
  // (DDC_FAR_OFF=1 in the environment keeps the direct sums: a diagnostic
  // switch for the tests)
  {
    const char* off = std::getenv("DDC_FAR_OFF");
    // a batch sums each molecule's own charges: the split pays only when one
    // of its molecules is large (the direct per-molecule sums of the
    // 256-globule batch, 1,952 spheres at most, take half the time of the
    // split, whose near lists hold most of each molecule)
    int largest = N;
    if (ctx->batch_init) {
      largest = 0;
      for (int k = 0; k < ctx->nmol; k++)
        largest = std::max(largest, ctx->h_off[k + 1] - ctx->h_off[k]);
    }
    ctx->far_on = largest >= kFarMinSpheres && G <= 640 && !(off && off[0] == '1');
    if (ctx->far_on) {
      const int YP = ctx->tbP.nylm;
      CK(ctx->farBT.ensure(sizeof(double) * YP * G));
      CK(ctx->farDT.ensure(sizeof(double) * 3 * YP * G));
      CK(ctx->farA.ensure(sizeof(double) * (size_t)YP * N));
      CK(launch_far_tables(L, ctx->tbP, ctx->grid.as<double4>(), G, ctx->farBT.as<double>(),
                           ctx->farDT.as<double>()));
    }
    // the field of zeta at the nuclei of one large molecule in the mixed
    // flow: spheres grouped for the multipole far field (DDC_ZFAR_OFF=1, or
    // DDC_FAR_OFF=1, keeps the direct FP32 pair sums)
    const char* zoff = std::getenv("DDC_ZFAR_OFF");
    ctx->zfar_on = ctx->zg_on && ctx->prm.precision == DDC_PREC_MIXED && ctx->prm.igrad &&
                   !(off && off[0] == '1') && !(zoff && zoff[0] == '1');
    if (ctx->zfar_on) {
      CK(ctx->zg_npt.ensure(sizeof(int) * (N + 1)));
      CK(ctx->zg_ptr.ensure(sizeof(int) * (N + 1)));
      const size_t tb = zgroups_scan_bytes(N);
      CK(ctx->zg_tmp.ensure(tb));
      ZGroups& z = ctx->zg;
      z.gnpt = ctx->zg_npt.as<int>();
      z.gptr = ctx->zg_ptr.as<int>();
      CK(launch_zgroups_points(L, ctx->cavoff.as<int>(), z, ctx->zg_tmp.p, tb));
      CK(ctx->zg_M.ensure(sizeof(float2) * zgroups_moment_count(z)));
      CK(ctx->zg_pk.ensure(sizeof(float4) * std::max(ctx->ncav, 1)));
      CK(ctx->zg_scr.ensure(sizeof(double) * 3 * (size_t)zgroups_nchunk(z) * N));
    }
  }
  CKI(sync(ctx));
  ctx->ready = true;
  return DDC_OK;
}

// ---------------------------------------------------------------------------
// the operators' two dense contractions, on the context's stream
// ---------------------------------------------------------------------------
// y(lm,i) = alpha sum_n bw(lm,n) pot(n,i): intrhs over every sphere
// (matvec.f90:131-135, bw = w_n Y_lm(s_n))
int gemm_proj(ddc_ctx* ctx, double alpha, const double* pot, double* y) {
  CK(launch_dgemm_nn(ctx->L(), ctx->nylm, ctx->nsph, ctx->ngrid, alpha, ctx->bw.as<double>(),
                     ctx->nylm, pot, ctx->ngrid, y, ctx->nylm, ctx->sweep));
  return DDC_OK;
}
// projection of the FP32 field (rows ldp_f apart) into the FP64 vector y
int gemm_proj_f32(ddc_ctx* ctx, float alpha, const float* pot, double* y) {
  if (ctx->tc.on)
    CK(launch_proj_tc(ctx->L(), ctx->tc, alpha, y, ctx->sweep));
  else
    CK(launch_proj_f32_simt(ctx->L(), ctx->nylm, ctx->nsph, ctx->ngrid, alpha,
                            ctx->bw_f.as<float>(), pot, ctx->ldp_f, y));
  return DDC_OK;
}
// xi(n,i) = sum_lm basis(lm,n) s(lm,i)   (matvec.f90:189-204)
int gemm_xi(ddc_ctx* ctx, const double* s, double* xig) {
  CK(launch_dgemm_nn(ctx->L(), ctx->ngrid, ctx->nsph, ctx->nylm, 1.0, ctx->basisT.as<double>(),
                     ctx->ngrid, s, ctx->nylm, xig, ctx->ngrid, ctx->sweep));
  return DDC_OK;
}
// FP32 xi of the FP64 vector s
int gemm_xi_f32(ddc_ctx* ctx, const double* s, float* xig) {
  if (ctx->tc.on)
    CK(launch_xi_tc(ctx->L(), ctx->tc, s, xig, ctx->sweep));
  else
    CK(launch_xi_f32_simt(ctx->L(), ctx->nylm, ctx->nsph, ctx->ngrid, ctx->basis_f.as<float>(),
                          s, xig));
  return DDC_OK;
}

// ---------------------------------------------------------------------------
// operators on device vectors
// ---------------------------------------------------------------------------
int op_lx(ddc_ctx* ctx, const double* x, double* y) {
  DevGeo g = ctx->geo();
  {
    // the lx part of the fused pass (one value per triple), then the sums
    // per grid point
    StageScope sc(ctx, ST_LX_POT);
    CK(launch_lx_vals(ctx->L(), ctx->tb, g, x, ctx->xk.p, ctx->tval.as<double>(), false));
    CK(launch_lx_gather(ctx->L(), g, ctx->tval.as<double>(), ctx->pot.as<double>()));
  }
  StageScope sc(ctx, ST_PROJ);
  // y = -Bw pot   (intrhs then negate, matvec.f90:131-135)
  return gemm_proj(ctx, -1.0, ctx->pot.as<double>(), y);
}
int op_xi(ddc_ctx* ctx, const double* x, double* xig) {
  // xi(n,i) = sum_lm basis(lm,n) x(lm,i)   (matvec.f90:189-204)
  StageScope sc(ctx, ST_XI);
  return gemm_xi(ctx, x, xig);
}
int op_lstarx(ddc_ctx* ctx, const double* x, double* y) {
  CKI(op_xi(ctx, x, ctx->xig.as<double>()));
  StageScope sc(ctx, ST_LSTARX);
  CK(launch_lstarx_acc(ctx->L(), ctx->tb, ctx->geo(), ctx->xig.as<double>(), y));
  return DDC_OK;
}

// FP32 operators of the mixed-precision path (vectors stay FP64)
int op_lx_f32(ddc_ctx* ctx, const double* x, double* y) {
  {
    StageScope sc(ctx, ST_LX_POT);
    DevGeo g = ctx->geo();
    CK(launch_lx_vals_f32(ctx->L(), ctx->tb, g, x, ctx->xk.p, ctx->tval.as<float>()));
    CK(launch_lx_gather_f32(ctx->L(), g, ctx->tval.as<float>(), ctx->pot_f.as<float>(),
                            ctx->ldp_f));
  }
  StageScope sc(ctx, ST_PROJ);
  return gemm_proj_f32(ctx, -1.f, ctx->pot_f.as<float>(), y);
}
int op_lstarx_f32(ddc_ctx* ctx, const double* x, double* y) {
  {
    StageScope sc(ctx, ST_XI);
    CKI(gemm_xi_f32(ctx, x, ctx->xi_f.as<float>()));
  }
  StageScope sc(ctx, ST_LSTARX);
  CK(launch_lstarx_acc_f32(ctx->L(), ctx->tb, ctx->geo(), ctx->xi_f.as<float>(), y));
  return DDC_OK;
}

// y = L x and z = L* s (off-diagonal parts) from one pass over the triples
int op_pair(ddc_ctx* ctx, const double* x, double* y, const double* s, double* z) {
  DevGeo g = ctx->geo();
  CKI(op_xi(ctx, s, ctx->xig.as<double>()));
  {
    StageScope sc(ctx, ST_LXS);
    CK(launch_lxs(ctx->L(), ctx->tb, g, x, ctx->xig.as<double>(), ctx->xk.p,
                  ctx->tval.as<double>(), z));
  }
  {
    StageScope sc(ctx, ST_GATHER);
    CK(launch_lx_gather(ctx->L(), g, ctx->tval.as<double>(), ctx->pot.as<double>()));
  }
  StageScope sc(ctx, ST_PROJ);
  return gemm_proj(ctx, -1.0, ctx->pot.as<double>(), y);
}
int op_pair_f32(ddc_ctx* ctx, const double* x, double* y, const double* s, double* z) {
  DevGeo g = ctx->geo();
  {
    StageScope sc(ctx, ST_XI);
    CKI(gemm_xi_f32(ctx, s, ctx->xi_f.as<float>()));
  }
  {
    StageScope sc(ctx, ST_LXS);
    CK(launch_lxs_f32(ctx->L(), ctx->tb, g, x, ctx->xi_f.as<float>(), ctx->xk.p,
                      ctx->tval.as<float>(), z));
  }
  {
    StageScope sc(ctx, ST_GATHER);
    CK(launch_lx_gather_f32(ctx->L(), g, ctx->tval.as<float>(), ctx->pot_f.as<float>(),
                            ctx->ldp_f));
  }
  StageScope sc(ctx, ST_PROJ);
  return gemm_proj_f32(ctx, -1.f, ctx->pot_f.as<float>(), y);
}

// gjinv (jacobi_diis.f90:272-360): Gauss-Jordan, full pivoting, one rhs.
bool gjinv(int n, std::vector<double>& a, std::vector<double>& b) {
  std::vector<int> indxc(n + 1), indxr(n + 1), piv(n + 1, 0);
  auto A = [&](int j, int k) -> double& { return a[(size_t)(k - 1) * n + (j - 1)]; };
  int irow = 0, icol = 0;
  for (int i = 1; i <= n; i++) {
    double big = 0.0;
    for (int j = 1; j <= n; j++)
      if (piv[j] != 1)
        for (int k = 1; k <= n; k++)
          if (piv[k] == 0 && std::fabs(A(j, k)) > big) {
            big = std::fabs(A(j, k));
            irow = j;
            icol = k;
          }
    if (icol == 0) return false;
    piv[icol] += 1;
    if (piv[icol] > 1) return false;
    if (irow != icol) {
      for (int k = 1; k <= n; k++) std::swap(A(irow, k), A(icol, k));
      std::swap(b[irow - 1], b[icol - 1]);
    }
    indxr[i] = irow;
    indxc[i] = icol;
    if (A(icol, icol) == 0.0) return false;
    double pinv = 1.0 / A(icol, icol);
    A(icol, icol) = 1.0;
    for (int k = 1; k <= n; k++) A(icol, k) *= pinv;
    b[icol - 1] *= pinv;
    for (int j = 1; j <= n; j++)
      if (j != icol) {
        double dum = A(j, icol);
        A(j, icol) = 0.0;
        for (int k = 1; k <= n; k++) A(j, k) -= A(icol, k) * dum;
        b[j - 1] -= b[icol - 1] * dum;
      }
  }
  for (int j = n; j >= 1; j--)
    if (indxr[j] != indxc[j])
      for (int k = 1; k <= n; k++) std::swap(A(k, indxr[j]), A(k, indxc[j]));
  return true;
}

typedef int (*OpFn)(ddc_ctx*, const double*, double*);

// Work vectors of one solve: set 0 is the context's, set 1 the second set
// used when the direct and adjoint systems are solved together.
struct SolveBufs {
  double *y, *xn, *hx, *he, *r, *d, *e;
};
SolveBufs solve_bufs(ddc_ctx* ctx, int set) {
  if (set == 0)
    return SolveBufs{ctx->y.as<double>(),      ctx->xn.as<double>(),   ctx->hist_x.as<double>(),
                     ctx->hist_e.as<double>(), ctx->rres.as<double>(), ctx->dres.as<double>(),
                     ctx->eres.as<double>()};
  return SolveBufs{ctx->y2.as<double>(),      ctx->xn2.as<double>(),   ctx->hist_x2.as<double>(),
                   ctx->hist_e2.as<double>(), ctx->rres2.as<double>(), ctx->dres2.as<double>(),
                   ctx->eres2.as<double>()};
}

// jacobi_diis (jacobi_diis.f90:1-176), norm mode 4 (hnorm), as a resumable
// state: the caller applies the operator to x into y, then jd_step performs
// the rest of the iteration (Jacobi step, DIIS extrapolation, increment
// norm and convergence test).  x holds the initial guess on entry and the
// solution on exit (device).  The log of increment norms continues at
// inf->norms[*logpos].
struct JDState {
  const double* rhs = nullptr;
  double* x = nullptr;
  double tol = 0.0;
  int max_iter = 0;
  double *y = nullptr, *hx = nullptr, *he = nullptr, *xjac = nullptr;
  std::vector<double> B;
  std::vector<int> map;
  int lenb = 0, nmat = 1, it = 0, restarts = 0;
  double rms = 0.0;
  bool done = false, ok = false;
  bool f32 = false;  // history vectors in FP32 (inner solves of the mixed path)
  ddc_solve_info* inf = nullptr;
  int* logpos = nullptr;
  int set = 0;  // which device row / pinned row of the reductions (0 direct, 1 adjoint)
  // between the three host steps of an iteration (jd_a, jd_b, jd_c)
  int p_nm = 0;
  bool p_shift = false;
  std::vector<int> p_map;
  void* p_xnew = nullptr;
  // history slot k of hx / he in the history precision
  void* slot(double* base, int k, long long n) const {
    return reinterpret_cast<char*>(base) + (size_t)k * n * (f32 ? sizeof(float) : sizeof(double));
  }
};

// DIIS history length: the reference's ndiis (jacobi_diis.f90) for the FP64
// solves; at most kInnerDiis for the FP32 inner solves of the mixed
// refinement, whose Jacobi step and extrapolation read the whole history
// from HBM every iteration (20k workload: 15 instead of 25 entries keeps the
// 88 / 85 iterations and takes 6 ms off the 190 ms step)
constexpr int kInnerDiis = 15;
int jd_ndiis(const ddc_ctx* ctx, bool f32) {
  return f32 ? std::min(ctx->prm.ndiis, kInnerDiis) : ctx->prm.ndiis;
}

void jd_begin(ddc_ctx* ctx, JDState& s, const double* rhs, double* x, double tol, int max_iter,
              const SolveBufs& b, ddc_solve_info* inf, int* logpos, bool f32 = false,
              int set = 0) {
  s.set = set;
  const int ndiis = jd_ndiis(ctx, f32);
  s.rhs = rhs;
  s.x = x;
  s.tol = tol;
  s.max_iter = max_iter;
  s.y = b.y;
  s.hx = b.hx;
  s.he = b.he;
  s.xjac = b.xn;
  s.lenb = ndiis + 1;
  s.B.assign((size_t)s.lenb * s.lenb, 0.0);
  s.map.resize(std::max(ndiis, 1));
  for (int k = 0; k < (int)s.map.size(); k++) s.map[k] = k;
  s.nmat = 1;
  s.it = 0;
  s.restarts = 0;
  s.rms = 0.0;
  s.ok = false;
  s.done = max_iter <= 0;
  s.f32 = f32;
  s.inf = inf;
  s.logpos = logpos;
}

// One iteration after y = op(x) (jacobi_diis.f90:120-160 with diis
// :183-230), in three host steps so that two systems solved together share
// their synchronisations: jd_a launches the Jacobi step with the Gram row
// and queues the row's copy to pinned memory; jd_b (after a synchronisation)
// updates the bordered system (makeb), solves it (gjinv) and launches the
// extrapolation with the increment norm, its copy queued; jd_c (after a
// synchronisation) reads the norm and applies the stop test.
double* red_row(ddc_ctx* ctx, int set) { return ctx->red.as<double>() + set * (kMaxHist + 1); }
double* hred_row(ddc_ctx* ctx, int set) { return ctx->hred + set * (kMaxHist + 1); }

int jd_a(ddc_ctx* ctx, JDState& s) {
  const long long n = (long long)ctx->nsph * ctx->nylm;
  const int ndiis = jd_ndiis(ctx, s.f32);
  const int nblk = reduce_blocks();
  ++s.it;
  HistPtrs hist{};
  double* out = red_row(ctx, s.set);
  if (ndiis != 0) {
    const int phys_new = s.map[s.nmat - 1];
    int nm = s.nmat;
    std::vector<int> pmap = s.map;
    const bool shift = s.nmat >= ndiis;
    if (shift) {  // drop the 10 oldest (jacobi_diis.f90:196-205)
      std::vector<int> r(s.map.begin() + 10, s.map.end());
      r.insert(r.end(), s.map.begin(), s.map.begin() + 10);
      pmap = r;
      nm = s.nmat - 10;
    }
    hist.n = nm - 1;
    for (int k = 0; k < nm - 1; k++) hist.p[k] = s.slot(s.he, pmap[k], n);
    void* xnew = s.slot(s.hx, phys_new, n);
    void* enew = s.slot(s.he, phys_new, n);
    {
      StageScope sc(ctx, ST_JACOBI);
      int jblk = nblk;
      CK(launch_jacobi_step(ctx->L(), ctx->tb, n, s.rhs, s.y, s.x, xnew, enew, hist,
                            ctx->partials.as<double>(), nblk, s.f32, &jblk,
                            ctx->rcount.as<unsigned>(), out));
    }
    CK(cudaMemcpyAsync(hred_row(ctx, s.set), out, sizeof(double) * nm, cudaMemcpyDeviceToHost,
                       ctx->st));
    s.p_nm = nm;
    s.p_shift = shift;
    s.p_map = pmap;
    s.p_xnew = xnew;
  } else {
    hist.n = 0;
    StageScope sc(ctx, ST_JACOBI);
    CK(launch_jacobi_step(ctx->L(), ctx->tb, n, s.rhs, s.y, s.x, s.hx, s.he, hist,
                          ctx->partials.as<double>(), nblk, s.f32, nullptr,
                          ctx->rcount.as<unsigned>(), out));
  }
  return DDC_OK;
}

int jd_b(ddc_ctx* ctx, JDState& s) {
  const long long n = (long long)ctx->nsph * ctx->nylm;
  const int ndiis = jd_ndiis(ctx, s.f32);
  const int lenb = s.lenb;
  auto Bm = [&](int j, int k) -> double& { return s.B[(size_t)(k - 1) * lenb + (j - 1)]; };
  HistPtrs comb{};
  const void* xj = s.hx;
  double* out = red_row(ctx, s.set);
  if (ndiis != 0) {
    const double* row = hred_row(ctx, s.set);
    if (s.p_shift) {
      for (int j = 2; j <= s.nmat - 10; j++)
        for (int k = 2; k <= s.nmat - 10; k++) Bm(j, k) = Bm(j + 10, k + 10);
      s.map = s.p_map;
    }
    s.nmat = s.p_nm;
    // makeb (jacobi_diis.f90:232-270)
    if (s.nmat == 1) {
      Bm(1, 1) = 0.0;
      Bm(1, 2) = 1.0;
      Bm(2, 1) = 1.0;
      Bm(2, 2) = row[0];
    } else {
      Bm(s.nmat + 1, 1) = 1.0;
      Bm(1, s.nmat + 1) = 1.0;
      for (int i = 1; i <= s.nmat - 1; i++) {
        Bm(s.nmat + 1, i + 1) = row[i - 1];
        Bm(i + 1, s.nmat + 1) = row[i - 1];
      }
      Bm(s.nmat + 1, s.nmat + 1) = row[s.nmat - 1];
    }
    const int nmat1 = s.nmat + 1;
    std::vector<double> bloc((size_t)nmat1 * nmat1), cex(nmat1, 0.0);
    for (int k = 1; k <= nmat1; k++)
      for (int j = 1; j <= nmat1; j++) bloc[(size_t)(k - 1) * nmat1 + (j - 1)] = Bm(j, k);
    cex[0] = 1.0;
    if (gjinv(nmat1, bloc, cex)) {
      comb.n = s.nmat;
      for (int k = 0; k < s.nmat; k++) {
        comb.p[k] = s.slot(s.hx, s.map[k], n);
        comb.c[k] = cex[k + 1];
      }
      s.nmat = s.nmat + 1;
    } else {  // singular: restart the history (jacobi_diis.f90:214-217)
      s.nmat = 1;
      s.restarts++;
      comb.n = 0;
    }
    xj = s.p_xnew;
  }
  {
    StageScope sc(ctx, ST_COMBINE);
    CK(launch_diis_combine(ctx->L(), ctx->tb, n, comb, xj, s.x, ctx->partials.as<double>(),
                           reduce_blocks(), s.f32, ctx->rcount.as<unsigned>(), out));
  }
  CK(cudaMemcpyAsync(hred_row(ctx, s.set), out, sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->st));
  return DDC_OK;
}

int jd_c(ddc_ctx* ctx, JDState& s) {
  const double ss = hred_row(ctx, s.set)[0];
  s.rms = std::sqrt(ss / (double)std::max(ctx->nsph, 1));
  if (*s.logpos < 256) s.inf->norms[*s.logpos] = s.rms;
  ++*s.logpos;
  if (ctx->prm.iprint > 0) printf("  iter=%4d residual norm: %14.4E\n", *s.logpos, s.rms);
  if (!std::isfinite(s.rms)) {
    s.done = true;
    return fail(ctx, DDC_ERR_NUMERIC, "non-finite increment norm");
  }
  s.ok = s.rms < s.tol;
  s.done = s.ok || s.it >= s.max_iter;
  return DDC_OK;
}

int jd_step(ddc_ctx* ctx, JDState& s) {
  CKI(jd_a(ctx, s));
  CKI(sync(ctx));
  CKI(jd_b(ctx, s));
  CKI(sync(ctx));
  return jd_c(ctx, s);
}

// FP64 solve: the reference's Jacobi/DIIS on the FP64 operator.
// Mixed solve: iterative refinement.  Each outer step forms in FP64 the
// residual r = rhs - L x and the Jacobi increment d = D^-1 r at x; its
// H-norm is the reference's convergence test (jacobi_diis.f90:143-150), so
// the solve stops exactly when the FP64 Jacobi increment is below
// 10^-iconv.  Otherwise the correction equation L e = r is solved with
// Jacobi/DIIS on the FP32 operator (from e = d, to 1e-4 relative) and x += e.
// A SolveTask is one such solve as a resumable state; solve_tasks advances
// one or two of them, one operator application each per round.
enum OpKind { OP_NONE = 0, OP_F64 = 1, OP_F32 = 2 };
struct SolveTask {
  bool adjoint = false, mixed = false;
  const double* rhs = nullptr;
  double* x = nullptr;
  ddc_solve_info* inf = nullptr;
  SolveBufs b{};
  double tol = 0.0, t0 = 0.0, last = 0.0;
  int phase = 0;  // mixed: 0 = FP64 residual at x next, 1 = inner solve running
  JDState jd;
  int logpos = 0, its = 0, restarts = 0, budget = 0, outer = 0;
  bool done = false, ok = false;
  // mixed, from the reference or the zero start: the first residual (at a
  // start that is never converged) comes from the FP32 operator, like the
  // inner iterations; the convergence test runs from the second refinement on
  bool f32_first = false;
  int set = 0;  // work-vector set and reduction row (0 direct, 1 adjoint)
};

void task_begin(ddc_ctx* ctx, SolveTask& t, bool adjoint, const double* rhs, double* x,
                ddc_solve_info* inf, int set) {
  t.adjoint = adjoint;
  t.mixed = ctx->prm.precision == DDC_PREC_MIXED;
  t.rhs = rhs;
  t.x = x;
  t.inf = inf;
  memset(inf, 0, sizeof(*inf));
  t.b = solve_bufs(ctx, set);
  t.set = set;
  t.tol = std::pow(10.0, -(double)ctx->prm.iconv);
  t.t0 = now_s();
  t.phase = 0;
  t.logpos = t.its = t.restarts = t.outer = 0;
  t.budget = ctx->prm.max_iter;
  t.last = 0.0;
  t.done = t.ok = false;
  t.f32_first = t.mixed && !ctx->guess_preset &&
                (ctx->prm.guess == DDC_GUESS_REFERENCE || ctx->prm.guess == DDC_GUESS_ZERO);
  if (!t.mixed)
    jd_begin(ctx, t.jd, rhs, x, t.tol, ctx->prm.max_iter, t.b, inf, &t.logpos, false, set);
  if (!t.mixed && t.jd.done) t.done = true;
}

// operator application the task needs next: kind, input, output
OpKind task_next(const SolveTask& t, const double** in, double** out) {
  if (t.done) return OP_NONE;
  if (!t.mixed || t.phase == 1) {
    *in = t.jd.x;
    *out = t.jd.y;
    return t.mixed ? OP_F32 : OP_F64;
  }
  *in = t.x;
  *out = t.b.y;
  return t.f32_first && t.outer == 0 ? OP_F32 : OP_F64;
}

// the task's next step is a Jacobi/DIIS iteration (FP64 solve, or an inner
// solve of the mixed refinement)
bool task_in_jd(const SolveTask& t) { return !t.mixed || t.phase == 1; }

// the task's bookkeeping after a Jacobi/DIIS iteration
int task_after_jd(ddc_ctx* ctx, SolveTask& t) {
  if (!t.jd.done) return DDC_OK;
  if (!t.mixed) {
    t.done = true;
    t.ok = t.jd.ok;
    t.its = t.jd.ok ? t.jd.it : ctx->prm.max_iter;
    t.restarts += t.jd.restarts;
    t.last = t.jd.rms;
    return DDC_OK;
  }
  const long long n = (long long)ctx->nsph * ctx->nylm;
  const int done = t.jd.ok ? t.jd.it : t.jd.max_iter;
  t.its += done;
  t.budget -= done;
  t.restarts += t.jd.restarts;
  CK(launch_axpy(ctx->L(), n, 1.0, t.b.e, t.x));
  t.phase = 0;
  if (t.outer >= 64) t.done = true;
  return DDC_OK;
}

int task_after(ddc_ctx* ctx, SolveTask& t) {
  if (task_in_jd(t)) {
    CKI(jd_step(ctx, t.jd));
    return task_after_jd(ctx, t);
  }
  const long long n = (long long)ctx->nsph * ctx->nylm;
  // phase 0: y = L x in FP64 is ready
  ++t.outer;
  {
    StageScope sc(ctx, ST_JACOBI);
    CK(launch_residual(ctx->L(), ctx->tb, n, t.rhs, t.b.y, t.x, t.b.r, t.b.d,
                       ctx->partials.as<double>(), reduce_blocks()));
  }
  double ss = 0.0;
  CKI(reduce_to_host(ctx, 1, &ss));
  t.last = std::sqrt(ss / (double)std::max(ctx->nsph, 1));
  const bool f32_res = t.f32_first && t.outer == 1;
  if (ctx->prm.iprint > 0)
    printf("  refinement %d: %s increment norm %14.4E\n", t.outer, f32_res ? "FP32" : "FP64",
           t.last);
  if (!std::isfinite(t.last)) {
    t.done = true;
    return fail(ctx, DDC_ERR_NUMERIC, "non-finite increment norm");
  }
  if (t.last < t.tol && !f32_res) {
    t.done = t.ok = true;
    return DDC_OK;
  }
  if (t.budget <= 0) {
    t.done = true;
    return DDC_OK;
  }
  // correction: (D + O32) e = r from e = D^-1 r
  CK(cudaMemcpyAsync(t.b.e, t.b.d, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
  // Each inner solve reduces its increment by rho (floor 0.3 tol).  Every
  // restart of the inner DIIS costs about ten iterations before the
  // extrapolation has a subspace again, so the split between the two inner
  // solves matters: at the 20,000-sphere workload rho = 1e-5 takes 88 / 86
  // iterations, 3e-5 86 / 80, 1e-4 80 / 79 (Esolv 2e-10 from the FP64
  // oracle; at most 3.9e-10 over eight smaller molecules, as with 1e-5), and
  // 3e-4 84 / 71 but 1.7e-9 on the 600-sphere configuration.
  // The correction is wanted to 1e-4 relative: FP32 history vectors suffice.
  const double rho = 1e-4;
  const double itol = std::max(rho * t.last, 0.3 * t.tol);
  jd_begin(ctx, t.jd, t.b.r, t.b.e, itol, t.budget, t.b, t.inf, &t.logpos, true, t.set);
  t.phase = 1;
  return DDC_OK;
}

int op_single(ddc_ctx* ctx, OpKind k, bool adjoint, const double* in, double* out) {
  if (k == OP_F64) return adjoint ? op_lstarx(ctx, in, out) : op_lx(ctx, in, out);
  return adjoint ? op_lstarx_f32(ctx, in, out) : op_lx_f32(ctx, in, out);
}

// Advance the tasks in lockstep.  When a direct and an adjoint task need an
// operator of the same precision in the same round, both come from one
// fused pass over the triples (op_pair / op_pair_f32).
int solve_tasks(ddc_ctx* ctx, SolveTask* t, int nt) {
  for (;;) {
    const double* in[2] = {nullptr, nullptr};
    double* out[2] = {nullptr, nullptr};
    OpKind k[2] = {OP_NONE, OP_NONE};
    int active = 0;
    for (int q = 0; q < nt; q++) {
      k[q] = task_next(t[q], &in[q], &out[q]);
      if (k[q] != OP_NONE) active++;
    }
    if (!active) break;
    // A task that needs an FP64 step (mixed refinement) while the other
    // runs FP32 inner iterations waits a round: the other reaches its own
    // FP64 step or finishes, and the FP64 steps then share a fused pass.
    // This only reorders the tasks' rounds; each keeps its own arithmetic.
    if (nt == 2 && k[0] != OP_NONE && k[1] != OP_NONE && k[0] != k[1]) {
      const int wait = k[0] == OP_F64 ? 0 : 1;
      k[wait] = OP_NONE;
    }
    if (nt == 2 && k[0] != OP_NONE && k[0] == k[1] && t[0].adjoint != t[1].adjoint) {
      const int dq = t[0].adjoint ? 1 : 0, aq = 1 - dq;
      if (k[0] == OP_F64) CKI(op_pair(ctx, in[dq], out[dq], in[aq], out[aq]));
      else CKI(op_pair_f32(ctx, in[dq], out[dq], in[aq], out[aq]));
    } else {
      for (int q = 0; q < nt; q++)
        if (k[q] != OP_NONE) CKI(op_single(ctx, k[q], t[q].adjoint, in[q], out[q]));
    }
    if (nt == 2 && k[0] != OP_NONE && k[1] != OP_NONE && task_in_jd(t[0]) && task_in_jd(t[1])) {
      // both systems take a Jacobi/DIIS iteration: one synchronisation for
      // both Gram rows and one for both increment norms (each system keeps
      // its own state, history and reduction row)
      CKI(jd_a(ctx, t[0].jd));
      CKI(jd_a(ctx, t[1].jd));
      CKI(sync(ctx));
      CKI(jd_b(ctx, t[0].jd));
      CKI(jd_b(ctx, t[1].jd));
      CKI(sync(ctx));
      CKI(jd_c(ctx, t[0].jd));
      CKI(jd_c(ctx, t[1].jd));
      CKI(task_after_jd(ctx, t[0]));
      CKI(task_after_jd(ctx, t[1]));
    } else {
      for (int q = 0; q < nt; q++)
        if (k[q] != OP_NONE) CKI(task_after(ctx, t[q]));
    }
  }
  int rc = DDC_OK;
  for (int q = 0; q < nt; q++) {
    ddc_solve_info* inf = t[q].inf;
    inf->iterations = t[q].its;
    inf->refinements = t[q].mixed ? t[q].outer : 0;
    inf->converged = t[q].ok ? 1 : 0;
    inf->diis_restarts = t[q].restarts;
    inf->final_norm = t[q].last;
    inf->seconds = now_s() - t[q].t0;
    if (!t[q].ok && rc == DDC_OK)
      rc = fail(ctx, DDC_ERR_NOCONV, t[q].adjoint ? "adjoint ddCOSMO did not converge"
                                                  : "ddCOSMO did not converge");
  }
  return rc;
}

int solve(ddc_ctx* ctx, bool adjoint, const double* rhs, double* x, ddc_solve_info* info) {
  ddc_solve_info loc{};
  SolveTask t;
  task_begin(ctx, t, adjoint, rhs, x, info ? info : &loc, 0);
  return solve_tasks(ctx, &t, 1);
}

int need_ready(ddc_ctx* ctx) {
  if (!ctx) return DDC_ERR_PARAM;
  if (!ctx->ready) return fail(ctx, DDC_ERR_STATE, "context not initialised (call ddc_init)");
  return DDC_OK;
}

// dot product on device, deterministic
int dot_dev(ddc_ctx* ctx, long long n, const double* a, const double* b, double* out) {
  CK(launch_dot_partial(ctx->L(), n, a, b, ctx->partials.as<double>(), reduce_blocks()));
  return reduce_to_host(ctx, 1, out);
}

// Solute potential (and, with ef, field) at the context's cavity points from
// charges q at its sphere centres (mkrhs.f90:102-114, main.f90:241): near /
// far split for large systems, direct sums otherwise.  trange: per-target
// source ranges of a batch (direct path); the split uses the molecule ranges.
int solute_pot_field(ddc_ctx* ctx, const double* q, double* phi, double* ef, const int2* trange) {
  const int N = ctx->nsph, NC = ctx->ncav;
  StageScope sc(ctx, ST_COULOMB);
  if (ctx->far_on) {
    CK(launch_far_pot_field(ctx->L(), ctx->tbP, N, ctx->ngrid, ctx->sph.as<double4>(), q,
                            ctx->mrange_ptr(), kFarRho, ctx->cavoff.as<int>(),
                            ctx->cavpt.as<int>(), ctx->ccav.as<double>(), ctx->farBT.as<double>(),
                            ctx->farDT.as<double>(), ctx->farA.as<double>(), phi, ef,
                            ctx->zg_on ? &ctx->zg : nullptr));
  } else if (ef) {
    CK(launch_coulomb_pot_field(ctx->L(), N, q, ctx->cx.as<double>(), ctx->cy.as<double>(),
                                ctx->cz.as<double>(), NC, ctx->ccav.as<double>(), phi, ef,
                                trange));
  } else {
    CK(launch_coulomb_pot(ctx->L(), N, q, ctx->cx.as<double>(), ctx->cy.as<double>(),
                          ctx->cz.as<double>(), NC, ctx->ccav.as<double>(), phi, trange));
  }
  return DDC_OK;
}

// right-hand side of the direct solve from the cavity potential: wghpot and
// intrhs (cosmo.f90:104-117)
int direct_rhs(ddc_ctx* ctx, const double* phi, double* rhs) {
  CK(ctx->gbuf.ensure(sizeof(double) * std::max<long long>((long long)ctx->nsph * ctx->ngrid, 1)));
  StageScope sc(ctx, ST_RHS);
  CK(launch_wghpot(ctx->L(), ctx->geo(), phi, ctx->gbuf.as<double>()));
  CK(launch_dgemm_nn(ctx->L(), ctx->nylm, ctx->nsph, ctx->ngrid, 1.0, ctx->bw.as<double>(),
                     ctx->nylm, ctx->gbuf.as<double>(), ctx->ngrid, rhs, ctx->nylm));
  return DDC_OK;
}

// cosmo on device vectors: phi (ncav) or glm -> sigma
int cosmo_dev(ddc_ctx* ctx, int star, int cart, const double* phi, const double* glm,
              const double* psi, double* sigma, double* esolv, ddc_solve_info* info) {
  const long long n = (long long)ctx->nsph * ctx->nylm;
  const int gmode = ctx->prm.guess == DDC_GUESS_ZERO ? 1 : 0;
  // the start is the caller's (USER) or was set by the energy+force flow
  const bool keep = ctx->prm.guess == DDC_GUESS_USER || ctx->guess_preset;
  if (ctx->prm.guess == DDC_GUESS_LEARNED && !ctx->guess_preset)
    return fail(ctx, DDC_ERR_PARAM,
                "the learned guess is formed by ddc_energy_forces / ddc_batch_energy_forces");
  if (!star) {
    double* rhs = ctx->rhs.as<double>();
    if (cart) {
      CKI(direct_rhs(ctx, phi, rhs));
    } else {
      CK(cudaMemcpyAsync(rhs, glm, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    }
    if (!keep) CK(launch_guess(ctx->L(), ctx->tb, n, rhs, sigma, gmode));
    CKI(solve(ctx, false, rhs, sigma, info));
    if (esolv) {
      double d = 0.0;
      CKI(dot_dev(ctx, n, sigma, psi, &d));
      *esolv = 0.5 * ((ctx->prm.eps - 1.0) / ctx->prm.eps) * d;
    }
  } else {
    if (!keep) CK(launch_guess(ctx->L(), ctx->tb, n, psi, sigma, gmode));
    CKI(solve(ctx, true, psi, sigma, info));
  }
  return DDC_OK;
}

// learned initial guesses x (direct) and s (adjoint, may be NULL) from the
// context's rhs g and psi: facl * rhs plus the model's correction
int learned_guess(ddc_ctx* ctx, const double* g, const double* psi, double* x, double* s) {
  ddc_guess* m = ctx->gmodel;
  if (!m) return fail(ctx, DDC_ERR_STATE, "DDC_GUESS_LEARNED needs a model (ddc_set_guess_model)");
  const int nin = guess_nfeat(m);
  CK(ctx->gfeat.ensure(sizeof(float) * std::max<long long>((long long)ctx->nsph * nin, 1)));
  CK(launch_guess_features(ctx->L(), ctx->nsph, ctx->nylm, nin, g, psi, ctx->sph.as<double4>(),
                           ctx->mrange_ptr(), ctx->gfeat.as<float>()));
  CK(guess_infer(ctx->L(), m, ctx->tb, ctx->nsph, ctx->gfeat.as<float>(), g, psi, x, s));
  return DDC_OK;
}

// forces_dd on device vectors (forces_dd.f90:91-164)
// xi_ready: xig already holds xi of s (the energy+force flow forms it first
// for zeta)
int forces_dev(ddc_ctx* ctx, const double* phi, const double* sigma, const double* s, double* fx,
               bool xi_ready = false) {
  if (!ctx->prm.igrad || !ctx->zi.p)
    return fail(ctx, DDC_ERR_STATE, "forces need igrad=1 at init (zi)");
  if (!xi_ready) CKI(op_xi(ctx, s, ctx->xig.as<double>()));
  {
    // u_chi(a, n) = sum over the neighbours b of chi(t) * intmlp(X_b): the
    // chi-weighted lx sum, per triple then per grid point
    StageScope sc(ctx, ST_UCHI);
    DevGeo g = ctx->geo();
    CK(launch_lx_vals(ctx->L(), ctx->tb, g, sigma, ctx->xk.p, ctx->tval.as<double>(), true));
    CK(launch_lx_gather(ctx->L(), g, ctx->tval.as<double>(), ctx->uchi.as<double>()));
  }
  const double fep = 0.5 * (ctx->prm.eps - 1.0) / ctx->prm.eps;
  CK(ctx->fxa.ensure(sizeof(double) * 3 * std::max(ctx->nsph, 1)));
  CK(ctx->fda.ensure(sizeof(double) * 3 * std::max<long long>(ctx->ntri, 1)));
  const int nlm = (ctx->prm.lmax + 1) * (ctx->prm.lmax + 2) / 2;
  CK(ctx->fvec.ensure(sizeof(double2) * 4 * nlm * std::max(ctx->nsph, 1)));
  StageScope sc(ctx, ST_FORCES);
  CK(launch_forces(ctx->L(), ctx->tb, ctx->geo(), sigma, ctx->xig.as<double>(),
                   ctx->uchi.as<double>(), phi, fep, fx, ctx->fxa.as<double>(),
                   ctx->fda.as<double>(), ctx->fvec.as<double2>()));
  return DDC_OK;
}

}  // namespace

// Batched Jacobi/DIIS: every molecule runs the reference's algorithm on its
// own segment of the concatenated vectors (own history, Gram matrix,
// restarts and convergence test); per iteration two kernels over element
// chunks do the Jacobi step and Gram row, then the bordered solve (the
// molecule's last chunk), the extrapolation and the norm for all molecules;
// a stopped molecule's chunks return at once.  iters receives the
// per-molecule iteration counts.
// One system of a batched solve: its right-hand side, iterate, operator
// output and per-molecule Jacobi/DIIS state on the device.  The state arrays
// of the two systems of a paired solve sit side by side in the same buffers
// (set 0, set 1).
struct BatchSys {
  bool adjoint = false;
  const double* rhs = nullptr;
  double* x = nullptr;
  double* y = nullptr;
  BatchState bs{};
  int* iters = nullptr;
  ddc_solve_info* inf = nullptr;
};

// f32: an inner solve of the mixed refinement (FP32 history of at most
// kInnerDiis vectors); status0 (host, or null: every non-empty molecule
// runs), tolk and maxk (host, or null: the parameters' tolerance and budget)
// give the molecules' starting status, tolerance and iteration budget.
int batch_setup(ddc_ctx* ctx, BatchSys& b, bool adjoint, const double* rhs, double* x,
                int* iters, ddc_solve_info* inf, int set, bool f32 = false,
                const int* status0 = nullptr, const double* tolk = nullptr,
                const int* maxk = nullptr) {
  const int nmol = ctx->nmol;
  const int nd = std::max(f32 ? std::min(ctx->prm.ndiis, kInnerDiis) : ctx->prm.ndiis, 11);
  if (ctx->prm.ndiis == 0) return fail(ctx, DDC_ERR_UNSUPPORTED, "batched solves need DIIS");
  std::vector<int> nmat(nmol, 1), slot((size_t)nmol * nd);
  for (int k = 0; k < nmol; k++)
    for (int j = 0; j < nd; j++) slot[(size_t)k * nd + j] = j;
  std::vector<int> status(nmol, 0);
  for (int k = 0; k < nmol; k++)
    if (ctx->h_off[k + 1] == ctx->h_off[k]) status[k] = 1;  // empty molecule
    else if (status0) status[k] = status0[k];
  const size_t lenb = nd + 1, lb2 = lenb * lenb;
  // room for both sets
  CK(ctx->b_nmat.ensure(sizeof(int) * 2 * nmol));
  CK(ctx->b_slot.ensure(sizeof(int) * 2 * nmol * nd));
  CK(ctx->b_B.ensure(sizeof(double) * 2 * nmol * lb2));
  CK(ctx->b_status.ensure(sizeof(int) * 2 * nmol));
  CK(ctx->b_iters.ensure(sizeof(int) * 2 * nmol));
  CK(ctx->b_restarts.ensure(sizeof(int) * 2 * nmol));
  CK(ctx->b_norm.ensure(sizeof(double) * 2 * nmol));
  // element chunks of each molecule (the same for both sets)
  std::vector<int> cfirst(nmol + 1, 0), cmol;
  for (int k = 0; k < nmol; k++) {
    const long long len = (long long)(ctx->h_off[k + 1] - ctx->h_off[k]) * ctx->nylm;
    const int nc = (int)((len + kBatchChunk - 1) / kBatchChunk);
    for (int c = 0; c < nc; c++) cmol.push_back(k);
    cfirst[k + 1] = cfirst[k] + nc;
  }
  const int nchunk = cfirst[nmol];
  CK(ctx->b_cmol.ensure(sizeof(int) * std::max(nchunk, 1)));
  CK(ctx->b_cfirst.ensure(sizeof(int) * (nmol + 1)));
  CK(ctx->b_part.ensure(sizeof(double) * 2 * (size_t)std::max(nchunk, 1) * (kMaxHist + 1)));
  CK(ctx->b_cnt.ensure(sizeof(unsigned) * 2 * nmol));
  CK(ctx->b_coef.ensure(sizeof(double) * 2 * (size_t)nmol * kMaxHist));
  CK(ctx->b_ext.ensure(sizeof(int) * 2 * nmol));
  BatchState& bs = b.bs;
  bs.nchunk = nchunk;
  bs.cmol = ctx->b_cmol.as<int>();
  bs.cfirst = ctx->b_cfirst.as<int>();
  bs.part = ctx->b_part.as<double>() + (size_t)set * std::max(nchunk, 1) * (kMaxHist + 1);
  bs.cnt = ctx->b_cnt.as<unsigned>() + (size_t)set * nmol;
  bs.coef = ctx->b_coef.as<double>() + (size_t)set * nmol * kMaxHist;
  bs.ext = ctx->b_ext.as<int>() + (size_t)set * nmol;
  if (nchunk)
    CK(cudaMemcpyAsync(ctx->b_cmol.p, cmol.data(), sizeof(int) * nchunk, cudaMemcpyHostToDevice,
                       ctx->st));
  CK(cudaMemcpyAsync(ctx->b_cfirst.p, cfirst.data(), sizeof(int) * (nmol + 1),
                     cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemsetAsync(bs.cnt, 0, sizeof(unsigned) * nmol, ctx->st));
  {
    std::vector<int> sphmol(ctx->nsph);
    for (int k = 0; k < nmol; k++)
      for (int i = ctx->h_off[k]; i < ctx->h_off[k + 1]; i++) sphmol[i] = k;
    CK(ctx->b_sphmol.ensure(sizeof(int) * std::max(ctx->nsph, 1)));
    CK(cudaMemcpyAsync(ctx->b_sphmol.p, sphmol.data(), sizeof(int) * ctx->nsph,
                       cudaMemcpyHostToDevice, ctx->st));
  }
  bs.nmol = nmol;
  bs.ndiis = nd;
  bs.max_iter = ctx->prm.max_iter;
  bs.tol = std::pow(10.0, -(double)ctx->prm.iconv);
  bs.n_total = (long long)ctx->nsph * ctx->nylm;
  bs.off = ctx->d_off.as<int>();
  bs.nmat = ctx->b_nmat.as<int>() + (size_t)set * nmol;
  bs.slot = ctx->b_slot.as<int>() + (size_t)set * nmol * nd;
  bs.B = ctx->b_B.as<double>() + (size_t)set * nmol * lb2;
  bs.status = ctx->b_status.as<int>() + (size_t)set * nmol;
  bs.iters = ctx->b_iters.as<int>() + (size_t)set * nmol;
  bs.restarts = ctx->b_restarts.as<int>() + (size_t)set * nmol;
  bs.norm = ctx->b_norm.as<double>() + (size_t)set * nmol;
  const SolveBufs sb = solve_bufs(ctx, set);
  bs.hx = sb.hx;
  bs.he = sb.he;
  bs.f32 = f32 ? 1 : 0;
  bs.tolk = nullptr;
  bs.maxk = nullptr;
  if (tolk) {
    CK(ctx->b_tolk.ensure(sizeof(double) * 2 * nmol));
    double* dt = ctx->b_tolk.as<double>() + (size_t)set * nmol;
    CK(cudaMemcpyAsync(dt, tolk, sizeof(double) * nmol, cudaMemcpyHostToDevice, ctx->st));
    bs.tolk = dt;
  }
  if (maxk) {
    CK(ctx->b_maxk.ensure(sizeof(int) * 2 * nmol));
    int* dm = ctx->b_maxk.as<int>() + (size_t)set * nmol;
    CK(cudaMemcpyAsync(dm, maxk, sizeof(int) * nmol, cudaMemcpyHostToDevice, ctx->st));
    bs.maxk = dm;
  }
  CK(cudaMemcpyAsync(bs.nmat, nmat.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(bs.slot, slot.data(), sizeof(int) * nmol * nd, cudaMemcpyHostToDevice,
                     ctx->st));
  CK(cudaMemsetAsync(bs.B, 0, sizeof(double) * nmol * lb2, ctx->st));
  CK(cudaMemcpyAsync(bs.status, status.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice,
                     ctx->st));
  CK(cudaMemsetAsync(bs.iters, 0, sizeof(int) * nmol, ctx->st));
  CK(cudaMemsetAsync(bs.restarts, 0, sizeof(int) * nmol, ctx->st));
  b.adjoint = adjoint;
  b.rhs = rhs;
  b.x = x;
  b.y = sb.y;
  b.iters = iters;
  b.inf = inf;
  // the host copy of status must not be read before these copies land
  CKI(sync(ctx));
  return DDC_OK;
}

// Copies one system's per-molecule results back and fills its report.
int batch_finish(ddc_ctx* ctx, const BatchSys& b, double t0) {
  const int nmol = ctx->nmol;
  std::vector<int> status(nmol), its(nmol), rst(nmol);
  std::vector<double> nrm(nmol);
  CK(cudaMemcpyAsync(status.data(), b.bs.status, sizeof(int) * nmol, cudaMemcpyDeviceToHost,
                     ctx->st));
  CK(cudaMemcpyAsync(its.data(), b.bs.iters, sizeof(int) * nmol, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(rst.data(), b.bs.restarts, sizeof(int) * nmol, cudaMemcpyDeviceToHost,
                     ctx->st));
  CK(cudaMemcpyAsync(nrm.data(), b.bs.norm, sizeof(double) * nmol, cudaMemcpyDeviceToHost,
                     ctx->st));
  CKI(sync(ctx));
  int maxit = 0, nfail = 0, restarts = 0;
  double worst = 0.0;
  for (int k = 0; k < nmol; k++) {
    if (b.iters) b.iters[k] = its[k];
    maxit = std::max(maxit, its[k]);
    restarts += rst[k];
    if (status[k] != 1) nfail++;
    if (ctx->h_off[k + 1] > ctx->h_off[k]) worst = std::max(worst, nrm[k]);
  }
  if (b.inf) {
    memset(b.inf, 0, sizeof(*b.inf));
    b.inf->iterations = maxit;
    b.inf->converged = nfail == 0;
    b.inf->diis_restarts = restarts;
    b.inf->final_norm = worst;
    b.inf->seconds = now_s() - t0;
  }
  if (nfail)
    return fail(ctx, DDC_ERR_NOCONV,
                std::to_string(nfail) + " molecule(s) did not converge" +
                    (b.adjoint ? " (adjoint)" : ""));
  return DDC_OK;
}

// Batched Jacobi/DIIS over one system, or over a direct and an adjoint
// system together (one fused L / L* pass per sweep).  A CUDA graph of
// `check` sweeps (operator kernels + the fused per-molecule DIIS kernels)
// is captured once and replayed until every molecule of every system has
// stopped; a stopped molecule's DIIS block returns at once, so extra sweeps
// are harmless.
int batch_sweeps(ddc_ctx* ctx, BatchSys* sys, int ns) {
  const int nmol = ctx->nmol;
  const bool f32 = sys[0].bs.f32 != 0;
  const int check = 4;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  CK(cudaStreamSynchronize(ctx->st));
  ctx->capturing = true;
  // the sweeps skip the spheres of molecules whose systems have all stopped
  ctx->sweep = SweepMask{ctx->b_sphmol.as<int>(), sys[0].bs.status,
                         ns == 2 ? sys[1].bs.status : nullptr};
  cudaError_t ce = cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal);
  int orc = DDC_OK;
  if (ce == cudaSuccess) {
    for (int r = 0; r < check && orc == DDC_OK; r++) {
      if (ns == 2) {
        const int dq = sys[0].adjoint ? 1 : 0, aq = 1 - dq;
        orc = f32 ? op_pair_f32(ctx, sys[dq].x, sys[dq].y, sys[aq].x, sys[aq].y)
                  : op_pair(ctx, sys[dq].x, sys[dq].y, sys[aq].x, sys[aq].y);
      } else {
        orc = op_single(ctx, f32 ? OP_F32 : OP_F64, sys[0].adjoint, sys[0].x, sys[0].y);
      }
      for (int q = 0; q < ns && orc == DDC_OK; q++)
        if (launch_batch_diis(ctx->L(), ctx->tb, sys[q].bs, sys[q].rhs, sys[q].y, sys[q].x) !=
            cudaSuccess)
          orc = DDC_ERR_CUDA;
    }
    cudaError_t ee = cudaStreamEndCapture(ctx->st, &graph);
    if (ce == cudaSuccess) ce = ee;
  }
  ctx->capturing = false;
  ctx->sweep = SweepMask{};
  if (orc != DDC_OK) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return orc;
  }
  CK(ce);
  CK(cudaGraphInstantiate(&exec, graph, 0));
  std::vector<int> status(nmol);
  int it = 0, active = 1;
  cudaError_t ge = cudaSuccess;
  while (it < ctx->prm.max_iter && active > 0) {
    {
      StageScope sc(ctx, ST_COMBINE);
      ge = cudaGraphLaunch(exec, ctx->st);
    }
    if (ge != cudaSuccess) break;
    it += check;
    active = 0;
    for (int q = 0; q < ns; q++) {
      CK(cudaMemcpyAsync(status.data(), sys[q].bs.status, sizeof(int) * nmol,
                         cudaMemcpyDeviceToHost, ctx->st));
      CKI(sync(ctx));
      for (int k = 0; k < nmol; k++) active += status[k] == 0;
    }
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  CK(ge);
  return DDC_OK;
}

int batch_run(ddc_ctx* ctx, BatchSys* sys, int ns) {
  const double t0 = now_s();
  CKI(batch_sweeps(ctx, sys, ns));
  int rc = DDC_OK;
  for (int q = 0; q < ns; q++) {
    const int r = batch_finish(ctx, sys[q], t0);
    if (r != DDC_OK && rc == DDC_OK) rc = r;
  }
  return rc;
}

// Mixed-precision batched solve: the single-molecule refinement (FP64
// residual and convergence test, inner FP32 Jacobi/DIIS solve of the
// correction to rho = 1e-4 of its increment, x += e) with every molecule on
// its own schedule, the molecules in lockstep per phase: one FP64 operator
// pass for all molecules still refining (converged ones are skipped), the
// batched residual with per-molecule norms, then one batched inner solve
// whose molecules each carry their own tolerance and remaining budget.
// sys[q].rhs / .x are the systems' right-hand sides and iterates.
int batch_run_mixed(ddc_ctx* ctx, BatchSys* sys, int ns) {
  const double t0 = now_s();
  const int nmol = ctx->nmol;
  const double tol = std::pow(10.0, -(double)ctx->prm.iconv);
  const bool f32_first = !ctx->guess_preset && (ctx->prm.guess == DDC_GUESS_REFERENCE ||
                                                 ctx->prm.guess == DDC_GUESS_ZERO);
  CK(ctx->b_run.ensure(sizeof(int) * 2 * nmol));
  CK(ctx->b_upd.ensure(sizeof(int) * 2 * nmol));
  CK(ctx->b_onorm.ensure(sizeof(double) * 2 * nmol));
  // per system and molecule: outer status (0 refining, 1 converged, 2 budget
  // spent, 3 non-finite), iterations, refinements, restarts, last norm
  std::vector<int> run(2 * nmol, 0), its(2 * nmol, 0), outer(2 * nmol, 0), rst(2 * nmol, 0);
  std::vector<double> last(2 * nmol, 0.0);
  for (int q = 0; q < ns; q++)
    for (int k = 0; k < nmol; k++)
      if (ctx->h_off[k + 1] == ctx->h_off[k]) run[q * nmol + k] = 1;
  int* drun = ctx->b_run.as<int>();
  int* dupd = ctx->b_upd.as<int>();
  double* dnorm = ctx->b_onorm.as<double>();
  BatchSys in[2];  // the inner systems: L e = r from e = d
  for (int round = 0; round < 64; round++) {
    int nrun = 0;
    for (int q = 0; q < ns; q++)
      for (int k = 0; k < nmol; k++) nrun += run[q * nmol + k] == 0;
    if (!nrun) break;
    CK(cudaMemcpyAsync(drun, run.data(), sizeof(int) * 2 * nmol, cudaMemcpyHostToDevice, ctx->st));
    // y = L x for the molecules still refining (FP32 at a reference or zero
    // start, whose first residual is never tested)
    const bool f32_res = f32_first && round == 0;
    ctx->sweep = SweepMask{ctx->b_sphmol.as<int>(), drun, ns == 2 ? drun + nmol : nullptr};
    int orc;
    if (ns == 2) {
      const int dq = sys[0].adjoint ? 1 : 0, aq = 1 - dq;
      const SolveBufs bd = solve_bufs(ctx, dq), ba = solve_bufs(ctx, aq);
      orc = f32_res ? op_pair_f32(ctx, sys[dq].x, bd.y, sys[aq].x, ba.y)
                    : op_pair(ctx, sys[dq].x, bd.y, sys[aq].x, ba.y);
    } else {
      orc = op_single(ctx, f32_res ? OP_F32 : OP_F64, sys[0].adjoint, sys[0].x,
                      solve_bufs(ctx, 0).y);
    }
    ctx->sweep = SweepMask{};
    CKI(orc);
    for (int q = 0; q < ns; q++) {
      const SolveBufs b = solve_bufs(ctx, q);
      StageScope sc(ctx, ST_JACOBI);
      CK(launch_batch_residual(ctx->L(), ctx->tb, sys[q].bs, drun + q * nmol, sys[q].rhs, b.y,
                               sys[q].x, b.r, b.d, b.e, dnorm + q * nmol));
    }
    std::vector<double> nrm(2 * nmol, 0.0);
    CK(cudaMemcpyAsync(nrm.data(), dnorm, sizeof(double) * 2 * nmol, cudaMemcpyDeviceToHost,
                       ctx->st));
    CKI(sync(ctx));
    // per molecule: converged, out of budget, or an inner solve
    std::vector<int> ist(2 * nmol, 1), maxk(2 * nmol, 1), upd(2 * nmol, 0);
    std::vector<double> tolk(2 * nmol, tol);
    int ninner = 0;
    for (int q = 0; q < ns; q++)
      for (int k = 0; k < nmol; k++) {
        const int j = q * nmol + k;
        if (run[j] != 0) continue;
        ++outer[j];
        last[j] = nrm[j];
        if (!std::isfinite(nrm[j])) {
          run[j] = 3;
        } else if (nrm[j] < tol && !f32_res) {
          run[j] = 1;
        } else if (its[j] >= ctx->prm.max_iter) {
          run[j] = 2;
        } else {
          ist[j] = 0;
          upd[j] = 1;
          maxk[j] = ctx->prm.max_iter - its[j];
          tolk[j] = std::max(1e-4 * nrm[j], 0.3 * tol);
          ++ninner;
        }
      }
    if (!ninner) break;
    for (int q = 0; q < ns; q++) {
      const SolveBufs b = solve_bufs(ctx, q);
      CKI(batch_setup(ctx, in[q], sys[q].adjoint, b.r, b.e, nullptr, nullptr, q, true,
                      ist.data() + q * nmol, tolk.data() + q * nmol, maxk.data() + q * nmol));
    }
    CKI(batch_sweeps(ctx, in, ns));
    // account the inner solves and apply their corrections
    CK(cudaMemcpyAsync(dupd, upd.data(), sizeof(int) * 2 * nmol, cudaMemcpyHostToDevice, ctx->st));
    std::vector<int> iit(2 * nmol, 0), irs(2 * nmol, 0);
    for (int q = 0; q < ns; q++) {
      CK(launch_batch_update(ctx->L(), in[q].bs, ctx->nylm, dupd + q * nmol,
                             solve_bufs(ctx, q).e, sys[q].x));
      CK(cudaMemcpyAsync(iit.data() + q * nmol, in[q].bs.iters, sizeof(int) * nmol,
                         cudaMemcpyDeviceToHost, ctx->st));
      CK(cudaMemcpyAsync(irs.data() + q * nmol, in[q].bs.restarts, sizeof(int) * nmol,
                         cudaMemcpyDeviceToHost, ctx->st));
    }
    CKI(sync(ctx));
    for (int j = 0; j < 2 * nmol; j++)
      if (upd[j]) {
        its[j] += iit[j];
        rst[j] += irs[j];
      }
  }
  int rc = DDC_OK;
  for (int q = 0; q < ns; q++) {
    int maxit = 0, maxout = 0, nfail = 0, restarts = 0;
    double worst = 0.0;
    for (int k = 0; k < nmol; k++) {
      const int j = q * nmol + k;
      if (sys[q].iters) sys[q].iters[k] = its[j];
      maxit = std::max(maxit, its[j]);
      maxout = std::max(maxout, outer[j]);
      restarts += rst[j];
      if (run[j] != 1 && ctx->h_off[k + 1] > ctx->h_off[k]) nfail++;
      if (ctx->h_off[k + 1] > ctx->h_off[k]) worst = std::max(worst, last[j]);
    }
    if (sys[q].inf) {
      memset(sys[q].inf, 0, sizeof(*sys[q].inf));
      sys[q].inf->iterations = maxit;
      sys[q].inf->refinements = maxout;
      sys[q].inf->converged = nfail == 0;
      sys[q].inf->diis_restarts = restarts;
      sys[q].inf->final_norm = worst;
      sys[q].inf->seconds = now_s() - t0;
    }
    if (nfail && rc == DDC_OK)
      rc = fail(ctx, DDC_ERR_NOCONV,
                std::to_string(nfail) + " molecule(s) did not converge" +
                    (sys[q].adjoint ? " (adjoint)" : ""));
  }
  return rc;
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int ddc_default_params(ddc_params* p) {
  if (!p) return DDC_ERR_PARAM;
  memset(p, 0, sizeof(*p));
  p->lmax = 6;
  p->ngrid = 110;
  p->iconv = 7;
  p->igrad = 1;
  p->eps = 78.3553;
  p->eta = 0.2;
  p->iprint = 0;
  p->max_iter = 200;
  p->ndiis = 25;
  p->precision = DDC_PREC_FP64;
  p->guess = DDC_GUESS_REFERENCE;
  p->device = 0;
  p->device_pointers = 0;
  p->pair_solves = 1;
  return DDC_OK;
}

const char* ddc_status_string(int s) {
  switch (s) {
    case DDC_OK: return "ok";
    case DDC_ERR_PARAM: return "invalid parameter";
    case DDC_ERR_STATE: return "invalid call order";
    case DDC_ERR_CUDA: return "CUDA error";
    case DDC_ERR_NOMEM: return "device allocation failed";
    case DDC_ERR_NOCONV: return "solver did not converge";
    case DDC_ERR_UNSUPPORTED: return "unsupported parameter";
    case DDC_ERR_NUMERIC: return "non-finite result";
    case DDC_ERR_CAPACITY:
      return "problem exceeds the fixed scratch of the allocation-free entry point";
    default: return "unknown status";
  }
}

int ddc_create(const ddc_params* p, ddc_ctx** out) {
  if (!p || !out) return DDC_ERR_PARAM;
  *out = nullptr;
  if (p->lmax < 0 || p->lmax > DDC_MAX_LMAX) return DDC_ERR_UNSUPPORTED;
  if (p->ngrid <= 0 || p->iconv < 0 || p->eps <= 0.0 || !(p->eta > 0.0 && p->eta <= 1.0) ||
      p->max_iter <= 0 || p->ndiis < 0 || p->ndiis > kMaxHist || (p->ndiis > 0 && p->ndiis <= 10))
    return DDC_ERR_PARAM;
  if (p->precision != DDC_PREC_FP64 && p->precision != DDC_PREC_MIXED) return DDC_ERR_PARAM;
  if (p->guess < DDC_GUESS_REFERENCE || p->guess > DDC_GUESS_LEARNED) return DDC_ERR_PARAM;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DDC_ERR_CUDA;
  if (p->device < 0 || p->device >= ndev) return DDC_ERR_PARAM;
  if (cudaSetDevice(p->device) != cudaSuccess) return DDC_ERR_CUDA;
  ddc_ctx* c = new ddc_ctx();
  c->prm = *p;
  if (p->stream) {
    c->st = (cudaStream_t)p->stream;
    c->own_stream = false;
  } else if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return DDC_ERR_CUDA;
  }
  *out = c;
  return DDC_OK;
}

int ddc_destroy(ddc_ctx* c) {
  if (!c) return DDC_OK;
  cudaSetDevice(c->prm.device);
  if (c->st) cudaStreamSynchronize(c->st);
  cudaStream_t st = c->own_stream ? c->st : nullptr;
  for (auto& pe : c->ev_pending) {
    cudaEventDestroy(pe.second.first);
    cudaEventDestroy(pe.second.second);
  }
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  tc_release(c->tc);
  if (c->hred) cudaFreeHost(c->hred);
  if (c->st2) cudaStreamSynchronize(c->st2);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->st2) cudaStreamDestroy(c->st2);
  delete c;
  if (st) cudaStreamDestroy(st);
  return DDC_OK;
}

const char* ddc_last_error(ddc_ctx* c) { return c ? c->err.c_str() : "null context"; }

long long ddc_launch_count(ddc_ctx* c) { return c ? c->launches : 0; }

int ddc_stage_count(void) { return ST_N; }
const char* ddc_stage_name(int k) {
  static const char* names[ST_N] = {"init",    "coulomb_pot", "rhs",       "lx_pot",
                                    "proj_gemm", "xi_gemm",   "lstarx",    "jacobi_step",
                                    "diis_combine", "reduce", "uchi_pot",  "forces",
                                    "zeta",    "efield",      "contract",  "lx_lstarx",
                                    "lx_gather"};
  return (k >= 0 && k < ST_N) ? names[k] : "";
}
int ddc_stage_times(ddc_ctx* c, double* ms, long long* calls) {
  if (!c) return DDC_ERR_PARAM;
  cudaSetDevice(c->prm.device);
  if (!c->ev_pending.empty()) {
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return DDC_ERR_CUDA;
    resolve_timers(c);
  }
  for (int k = 0; k < ST_N; k++) {
    if (ms) ms[k] = c->st_ms[k];
    if (calls) calls[k] = c->st_calls[k];
  }
  return DDC_OK;
}
int ddc_set_timed_stages(ddc_ctx* c, unsigned int mask) {
  if (!c) return DDC_ERR_PARAM;
  c->stage_mask = mask;
  return DDC_OK;
}
int ddc_reset_stage_times(ddc_ctx* c) {
  if (!c) return DDC_ERR_PARAM;
  cudaSetDevice(c->prm.device);
  if (!c->ev_pending.empty()) {
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return DDC_ERR_CUDA;
    resolve_timers(c);
  }
  for (int k = 0; k < ST_N; k++) {
    c->st_ms[k] = 0.0;
    c->st_calls[k] = 0;
  }
  return DDC_OK;
}

}  // extern "C"

// FMA throughput probe: 8 dependent chains per thread, 8 blocks of 256 per SM
static int fma_peak(int device, bool fp32, double* gflops) {
  if (!gflops) return DDC_ERR_PARAM;
  if (cudaSetDevice(device) != cudaSuccess) return DDC_ERR_CUDA;
  cudaDeviceProp pr;
  if (cudaGetDeviceProperties(&pr, device) != cudaSuccess) return DDC_ERR_CUDA;
  long long launches = 0;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return DDC_ERR_CUDA;
  Launch L{st, &launches};
  double* out = nullptr;
  cudaEvent_t a, b;
  cudaMalloc(&out, sizeof(double));
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int blocks = pr.multiProcessorCount * 8, iters = fp32 ? 8192 : 4096;
  auto run = [&](int it) {
    if (fp32) launch_fp32_probe(L, blocks, it, reinterpret_cast<float*>(out));
    else launch_fp64_probe(L, blocks, it, out);
  };
  run(64);  // warm up
  cudaEventRecord(a, st);
  run(iters);
  cudaEventRecord(b, st);
  cudaError_t e = cudaStreamSynchronize(st);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  cudaStreamDestroy(st);
  if (e != cudaSuccess || ms <= 0.f) return DDC_ERR_CUDA;
  double flops = 2.0 * 8.0 * (double)iters * blocks * 256.0;
  *gflops = flops / (ms * 1e-3) / 1e9;
  return DDC_OK;
}

extern "C" {
int ddc_fp64_peak(int device, double* gflops) { return fma_peak(device, false, gflops); }
int ddc_fp32_peak(int device, double* gflops) { return fma_peak(device, true, gflops); }

int ddc_init(ddc_ctx* ctx, int n, const double* x, const double* y, const double* z,
             const double* r) {
  if (!ctx) return DDC_ERR_PARAM;
  if (n < 0 || (n > 0 && (!x || !y || !z || !r))) return fail(ctx, DDC_ERR_PARAM, "bad input");
  cudaSetDevice(ctx->prm.device);
  std::vector<double4> hs(n);
  if (ctx->prm.device_pointers) {
    std::vector<double> hx(n), hy(n), hz(n), hr(n);
    if (n) {
      CK(cudaMemcpy(hx.data(), x, sizeof(double) * n, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(hy.data(), y, sizeof(double) * n, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(hz.data(), z, sizeof(double) * n, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(hr.data(), r, sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    for (int i = 0; i < n; i++) hs[i] = make_double4(hx[i], hy[i], hz[i], hr[i]);
  } else {
    for (int i = 0; i < n; i++) hs[i] = make_double4(x[i], y[i], z[i], r[i]);
  }
  for (int i = 0; i < n; i++)
    if (!(hs[i].w > 0.0)) return fail(ctx, DDC_ERR_PARAM, "radii must be positive");
  if (!ctx->batch_init) ctx->nmol = 1;
  ctx->have_flow = false;
  int rc;
  {
    StageScope sc(ctx, ST_INIT);
    rc = do_init(ctx, n, &hs, nullptr);
  }
  if (rc == DDC_OK) CKI(sync(ctx));
  return rc;
}

int ddc_sizes(ddc_ctx* ctx, int* nsph, int* ncav, int* nylm, int* ngrid) {
  CKI(need_ready(ctx));
  if (nsph) *nsph = ctx->nsph;
  if (ncav) *ncav = ctx->ncav;
  if (nylm) *nylm = ctx->nylm;
  if (ngrid) *ngrid = ctx->ngrid;
  return DDC_OK;
}

static int get_dev_array(ddc_ctx* ctx, double* out, const void* src, size_t count) {
  CKI(need_ready(ctx));
  if (!out) return fail(ctx, DDC_ERR_PARAM, "null output");
  if (count == 0) return DDC_OK;
  CK(cudaMemcpyAsync(out, src, sizeof(double) * count,
                     ctx->prm.device_pointers ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     ctx->st));
  return sync(ctx);
}

int ddc_get_ccav(ddc_ctx* ctx, double* ccav) {
  CKI(need_ready(ctx));
  return get_dev_array(ctx, ccav, ctx->ccav.p, 3 * (size_t)ctx->ncav);
}
int ddc_get_ui(ddc_ctx* ctx, double* ui) {
  CKI(need_ready(ctx));
  return get_dev_array(ctx, ui, ctx->ui.p, (size_t)ctx->nsph * ctx->ngrid);
}
int ddc_get_csph(ddc_ctx* ctx, double* csph) {
  CKI(need_ready(ctx));
  return get_dev_array(ctx, csph, ctx->csph.p, 3 * (size_t)ctx->nsph);
}
int ddc_get_grid(ddc_ctx* ctx, double* grid, double* w) {
  CKI(need_ready(ctx));
  for (int i = 0; i < ctx->ngrid; i++) {
    if (grid)
      for (int k = 0; k < 3; k++) grid[3 * i + k] = ctx->h_grid[4 * i + k];
    if (w) w[i] = ctx->h_grid[4 * i + 3];
  }
  return DDC_OK;
}

int ddc_mkrhs(ddc_ctx* ctx, int n, const double* charge, const double* x, const double* y,
              const double* z, int ncav, const double* ccav, double* phi, int nylm, double* psi) {
  if (!ctx) return DDC_ERR_PARAM;
  cudaSetDevice(ctx->prm.device);
  if (n < 0 || ncav < 0 || nylm <= 0) return fail(ctx, DDC_ERR_PARAM, "bad sizes");
  if (!ccav) {
    CKI(need_ready(ctx));
    if (ncav != ctx->ncav) return fail(ctx, DDC_ERR_PARAM, "ncav does not match the context");
  }
  const double *dq, *dx, *dy, *dz, *dc;
  CKI(stage_in(ctx, charge, n, ctx->in1, &dq));
  CKI(stage_in(ctx, x, n, ctx->in2, &dx));
  CKI(stage_in(ctx, y, n, ctx->in3, &dy));
  CKI(stage_in(ctx, z, n, ctx->in4, &dz));
  if (ccav) CKI(stage_in(ctx, ccav, 3 * (size_t)ncav, ctx->ef2, &dc));
  else dc = ctx->ccav.as<double>();
  double *dphi, *dpsi;
  CKI(out_ptr(ctx, phi, ncav, ctx->phi, &dphi));
  CKI(out_ptr(ctx, psi, (size_t)n * nylm, ctx->out1, &dpsi));
  CK(launch_coulomb_pot(ctx->L(), n, dq, dx, dy, dz, ncav, dc, dphi, nullptr));
  CK(launch_psi(ctx->L(), n, nylm, dq, dpsi));
  CKI(finish_out(ctx, phi, dphi, ncav));
  CKI(finish_out(ctx, psi, dpsi, (size_t)n * nylm));
  return sync(ctx);
}

int ddc_rhs(ddc_ctx* ctx, const double* phi, double* g) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  const double* dphi;
  CKI(stage_in(ctx, phi, ctx->ncav, ctx->in1, &dphi));
  double* dg;
  CKI(out_ptr(ctx, g, (size_t)ctx->nsph * ctx->nylm, ctx->out1, &dg));
  CK(ctx->gbuf.ensure(sizeof(double) * std::max<long long>((long long)ctx->nsph * ctx->ngrid, 1)));
  CK(launch_wghpot(ctx->L(), ctx->geo(), dphi, ctx->gbuf.as<double>()));
  CK(launch_dgemm_nn(ctx->L(), ctx->nylm, ctx->nsph, ctx->ngrid, 1.0, ctx->bw.as<double>(),
                     ctx->nylm, ctx->gbuf.as<double>(), ctx->ngrid, dg, ctx->nylm));
  CKI(finish_out(ctx, g, dg, (size_t)ctx->nsph * ctx->nylm));
  return sync(ctx);
}

int ddc_cosmo(ddc_ctx* ctx, int star, int cart, const double* phi, const double* glm,
              const double* psi, double* sigma, double* esolv, ddc_solve_info* info) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  if (!sigma) return fail(ctx, DDC_ERR_PARAM, "null sigma");
  const size_t nv = (size_t)ctx->nsph * ctx->nylm;
  const double *dphi = nullptr, *dglm = nullptr, *dpsi = nullptr;
  if (!star) {
    if (cart) CKI(stage_in(ctx, phi, ctx->ncav, ctx->in1, &dphi));
    else CKI(stage_in(ctx, glm, nv, ctx->in1, &dglm));
    if (esolv) CKI(stage_in(ctx, psi, nv, ctx->in2, &dpsi));
  } else {
    CKI(stage_in(ctx, psi, nv, ctx->in2, &dpsi));
  }
  double* dsig;
  if (ctx->prm.device_pointers) {
    dsig = sigma;
  } else {
    dsig = ctx->sigma.as<double>();
    if (ctx->prm.guess == DDC_GUESS_USER)
      CK(cudaMemcpyAsync(dsig, sigma, sizeof(double) * nv, cudaMemcpyHostToDevice, ctx->st));
  }
  int rc = cosmo_dev(ctx, star, cart, dphi, dglm, dpsi, dsig, star ? nullptr : esolv, info);
  if (rc != DDC_OK && rc != DDC_ERR_NOCONV) return rc;
  if (!ctx->prm.device_pointers)
    CK(cudaMemcpyAsync(sigma, dsig, sizeof(double) * nv, cudaMemcpyDeviceToHost, ctx->st));
  CKI(sync(ctx));
  return rc;
}

int ddc_forces_dd(ddc_ctx* ctx, const double* phi, const double* sigma, const double* s,
                  double* fx) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  const size_t nv = (size_t)ctx->nsph * ctx->nylm;
  const double *dphi, *dsig, *ds;
  CKI(stage_in(ctx, phi, ctx->ncav, ctx->in1, &dphi));
  CKI(stage_in(ctx, sigma, nv, ctx->in2, &dsig));
  CKI(stage_in(ctx, s, nv, ctx->in3, &ds));
  double* dfx;
  CKI(out_ptr(ctx, fx, 3 * (size_t)ctx->nsph, ctx->fx, &dfx));
  CKI(forces_dev(ctx, dphi, dsig, ds, dfx));
  CKI(finish_out(ctx, fx, dfx, 3 * (size_t)ctx->nsph));
  return sync(ctx);
}

static int mkxi_common(ddc_ctx* ctx, const double* s, double* out, double scale) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  const double* ds;
  CKI(stage_in(ctx, s, (size_t)ctx->nsph * ctx->nylm, ctx->in1, &ds));
  double* dout;
  CKI(out_ptr(ctx, out, ctx->ncav, ctx->zeta, &dout));
  CKI(op_xi(ctx, ds, ctx->xig.as<double>()));
  CK(launch_mkxi(ctx->L(), ctx->tb, ctx->geo(), ctx->xig.as<double>(), scale, dout));
  CKI(finish_out(ctx, out, dout, ctx->ncav));
  return sync(ctx);
}
int ddc_mkzeta(ddc_ctx* ctx, const double* s, double* zeta) {
  if (!ctx) return DDC_ERR_PARAM;
  return mkxi_common(ctx, s, zeta, 0.5 * ((ctx->prm.eps - 1.0) / ctx->prm.eps));
}
int ddc_mkxi(ddc_ctx* ctx, const double* s, double* xi) { return mkxi_common(ctx, s, xi, 1.0); }

int ddc_efld(ddc_ctx* ctx, int nsrc, const double* src, const double* csrc, int ntrg,
             const double* ctrg, double* ef) {
  if (!ctx) return DDC_ERR_PARAM;
  cudaSetDevice(ctx->prm.device);
  if (nsrc < 0 || ntrg < 0) return fail(ctx, DDC_ERR_PARAM, "bad sizes");
  auto ctx_coords = [&](int cnt, const double** out) -> int {
    CKI(need_ready(ctx));
    if (cnt == ctx->ncav) *out = ctx->ccav.as<double>();
    else if (cnt == ctx->nsph) *out = ctx->csph.as<double>();
    else return fail(ctx, DDC_ERR_PARAM, "NULL coordinates need ncav or nsph points");
    return DDC_OK;
  };
  const double *dsrc, *dcs, *dct;
  CKI(stage_in(ctx, src, nsrc, ctx->in1, &dsrc));
  if (csrc) CKI(stage_in(ctx, csrc, 3 * (size_t)nsrc, ctx->in2, &dcs));
  else CKI(ctx_coords(nsrc, &dcs));
  if (ctrg) CKI(stage_in(ctx, ctrg, 3 * (size_t)ntrg, ctx->in3, &dct));
  else CKI(ctx_coords(ntrg, &dct));
  double* def;
  CKI(out_ptr(ctx, ef, 3 * (size_t)ntrg, ctx->out1, &def));
  int nchunk = efield_chunks(nsrc, ntrg);
  CK(ctx->ef_scratch.ensure(sizeof(double) * 3 * (size_t)std::max(ntrg, 1) * nchunk));
  CK(launch_efield(ctx->L(), nsrc, dsrc, dcs, ntrg, dct, def, ctx->ef_scratch.as<double>(),
                   nchunk, nullptr));
  CKI(finish_out(ctx, ef, def, 3 * (size_t)ntrg));
  return sync(ctx);
}

int ddc_lx(ddc_ctx* ctx, const double* x, double* y) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  const size_t nv = (size_t)ctx->nsph * ctx->nylm;
  const double* dx;
  CKI(stage_in(ctx, x, nv, ctx->in1, &dx));
  double* dy;
  CKI(out_ptr(ctx, y, nv, ctx->out1, &dy));
  if (ctx->prm.precision == DDC_PREC_MIXED)
    CKI(op_lx_f32(ctx, dx, dy));
  else
    CKI(op_lx(ctx, dx, dy));
  CKI(finish_out(ctx, y, dy, nv));
  return sync(ctx);
}
int ddc_lstarx(ddc_ctx* ctx, const double* x, double* y) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  const size_t nv = (size_t)ctx->nsph * ctx->nylm;
  const double* dx;
  CKI(stage_in(ctx, x, nv, ctx->in1, &dx));
  double* dy;
  CKI(out_ptr(ctx, y, nv, ctx->out1, &dy));
  if (ctx->prm.precision == DDC_PREC_MIXED)
    CKI(op_lstarx_f32(ctx, dx, dy));
  else
    CKI(op_lstarx(ctx, dx, dy));
  CKI(finish_out(ctx, y, dy, nv));
  return sync(ctx);
}
int ddc_lx_lstarx(ddc_ctx* ctx, const double* x, double* y, const double* s, double* z) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  const size_t nv = (size_t)ctx->nsph * ctx->nylm;
  CK(ctx->tval.ensure(sizeof(double) * std::max<long long>(ctx->ntri, 1)));
  const double *dx, *ds;
  CKI(stage_in(ctx, x, nv, ctx->in1, &dx));
  CKI(stage_in(ctx, s, nv, ctx->in2, &ds));
  double *dy, *dz;
  CKI(out_ptr(ctx, y, nv, ctx->out1, &dy));
  if (ctx->prm.device_pointers) {
    dz = z;
  } else {
    CK(ctx->in3.ensure(sizeof(double) * std::max(nv, (size_t)1)));
    dz = ctx->in3.as<double>();
  }
  if (!dz) return fail(ctx, DDC_ERR_PARAM, "null output array");
  if (ctx->prm.precision == DDC_PREC_MIXED)
    CKI(op_pair_f32(ctx, dx, dy, ds, dz));
  else
    CKI(op_pair(ctx, dx, dy, ds, dz));
  CKI(finish_out(ctx, y, dy, nv));
  CKI(finish_out(ctx, z, dz, nv));
  return sync(ctx);
}
int ddc_ldm1x(ddc_ctx* ctx, const double* x, double* y) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  const size_t nv = (size_t)ctx->nsph * ctx->nylm;
  const double* dx;
  CKI(stage_in(ctx, x, nv, ctx->in1, &dx));
  double* dy;
  CKI(out_ptr(ctx, y, nv, ctx->out1, &dy));
  CK(launch_ldm1x(ctx->L(), ctx->tb, (long long)nv, dx, dy));
  CKI(finish_out(ctx, y, dy, nv));
  return sync(ctx);
}
int ddc_hnorm(ddc_ctx* ctx, const double* x, double* norm) {
  CKI(need_ready(ctx));
  cudaSetDevice(ctx->prm.device);
  if (!norm) return fail(ctx, DDC_ERR_PARAM, "null norm");
  const size_t nv = (size_t)ctx->nsph * ctx->nylm;
  const double* dx;
  CKI(stage_in(ctx, x, nv, ctx->in1, &dx));
  CK(launch_hnorm_partial(ctx->L(), ctx->tb, (long long)nv, dx, ctx->partials.as<double>(),
                          reduce_blocks()));
  double ss = 0.0;
  CKI(reduce_to_host(ctx, 1, &ss));
  *norm = std::sqrt(ss / (double)std::max(ctx->nsph, 1));
  return DDC_OK;
}

int ddc_energy_forces(ddc_ctx* ctx, int n, const double* charge, const double* x,
                      const double* y, const double* z, const double* rvdw, double* esolv,
                      double* sigma, double* s, double* fx, ddc_run_info* info) {
  if (!ctx || !esolv) return DDC_ERR_PARAM;
  cudaSetDevice(ctx->prm.device);
  ddc_run_info loc{};
  ddc_run_info* inf = info ? info : &loc;
  memset(inf, 0, sizeof(*inf));
  double t0 = now_s();
  CKI(ddc_init(ctx, n, x, y, z, rvdw));
  double t1 = now_s();
  inf->t_init = t1 - t0;
  const int N = ctx->nsph, NC = ctx->ncav;
  const size_t nv = (size_t)N * ctx->nylm;
  const double* dq;
  CKI(stage_in(ctx, charge, N, ctx->q, &dq));
  CK(ctx->phi.ensure(sizeof(double) * std::max(NC, 1)));
  double* dphi = ctx->phi.as<double>();
  double* dpsi = ctx->psi.as<double>();
  // mkrhs (mkrhs.f90:102-120) with the context's own centres and cavity; with
  // forces, the solute field at the cavity (main.f90:241-253) comes from the
  // same pass over the pairs
  if (ctx->prm.igrad) CK(ctx->ef1.ensure(sizeof(double) * 3 * std::max(NC, 1)));
  CKI(solute_pot_field(ctx, dq, dphi, ctx->prm.igrad ? ctx->ef1.as<double>() : nullptr,
                       nullptr));
  CK(launch_psi(ctx->L(), N, ctx->nylm, dq, dpsi));
  CKI(sync(ctx));
  double t2 = now_s();
  inf->t_mkrhs = t2 - t1;
  double* dsig = ctx->sigma.as<double>();
  double* ds = ctx->s.as<double>();
  if (ctx->prm.guess == DDC_GUESS_USER) {
    // sigma (and s) carry the initial guesses in, e.g. the previous frame's
    // solutions (the sigma slot of cosmo.f90:136-138, 174-176)
    if (!sigma || (ctx->prm.igrad && !s))
      return fail(ctx, DDC_ERR_PARAM, "user guess needs sigma and s on entry");
    const cudaMemcpyKind k =
        ctx->prm.device_pointers ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(dsig, sigma, sizeof(double) * nv, k, ctx->st));
    if (ctx->prm.igrad) CK(cudaMemcpyAsync(ds, s, sizeof(double) * nv, k, ctx->st));
  }
  const bool paired = ctx->prm.igrad && ctx->prm.pair_solves;
  if (paired) {
    // both systems at once: the adjoint right-hand side psi is known before
    // the direct solve, and each round applies L and L* in one fused pass
    double* rhs = ctx->rhs.as<double>();
    CKI(direct_rhs(ctx, dphi, rhs));
    if (ctx->prm.guess == DDC_GUESS_LEARNED) {
      CKI(learned_guess(ctx, rhs, dpsi, dsig, ds));
    } else if (ctx->prm.guess != DDC_GUESS_USER) {
      const int gmode = ctx->prm.guess == DDC_GUESS_ZERO ? 1 : 0;
      CK(launch_guess(ctx->L(), ctx->tb, (long long)nv, rhs, dsig, gmode));
      CK(launch_guess(ctx->L(), ctx->tb, (long long)nv, dpsi, ds, gmode));
    }
    SolveTask task[2];
    task_begin(ctx, task[0], false, rhs, dsig, &inf->direct, 0);
    task_begin(ctx, task[1], true, dpsi, ds, &inf->adjoint, 1);
    CKI(solve_tasks(ctx, task, 2));
    double d = 0.0;
    CKI(dot_dev(ctx, (long long)nv, dsig, dpsi, &d));
    *esolv = 0.5 * ((ctx->prm.eps - 1.0) / ctx->prm.eps) * d;
  } else {
    if (ctx->prm.guess == DDC_GUESS_LEARNED) {
      // both starts from the model before the solves (cosmo_dev recomputes
      // the same rhs and keeps them)
      CKI(direct_rhs(ctx, dphi, ctx->rhs.as<double>()));
      CKI(learned_guess(ctx, ctx->rhs.as<double>(), dpsi, dsig, ctx->prm.igrad ? ds : nullptr));
      ctx->guess_preset = true;
    }
    const int rc = cosmo_dev(ctx, 0, 1, dphi, nullptr, dpsi, dsig, esolv, &inf->direct);
    if (rc != DDC_OK || !ctx->prm.igrad) ctx->guess_preset = false;
    if (rc != DDC_OK) return rc;
  }
  double t3 = now_s();
  inf->t_direct = t3 - t2;
  double* dfx = nullptr;
  if (ctx->prm.igrad) {
    if (!paired) {
      const int rc = cosmo_dev(ctx, 1, 0, nullptr, nullptr, dpsi, ds, nullptr, &inf->adjoint);
      ctx->guess_preset = false;
      if (rc != DDC_OK) return rc;
    }
    double t4 = now_s();
    inf->t_adjoint = t4 - t3;
    CK(ctx->fx.ensure(sizeof(double) * 3 * std::max(N, 1)));
    dfx = ctx->fx.as<double>();
    // zeta first (ddmkzeta, ddcosmo.f90:1758-1806): the field of zeta at the
    // nuclei (main.f90:259-265) then runs on the second stream beside the
    // force kernels, which keep the FP64 pipe busy while it loads the FP32
    // (or FP64) pipe
    CKI(op_xi(ctx, ds, ctx->xig.as<double>()));
    CK(ctx->zeta.ensure(sizeof(double) * std::max(NC, 1)));
    double fep = 0.5 * ((ctx->prm.eps - 1.0) / ctx->prm.eps);
    {
      StageScope sc(ctx, ST_ZETA);
      CK(launch_mkxi(ctx->L(), ctx->tb, ctx->geo(), ctx->xig.as<double>(), fep,
                     ctx->zeta.as<double>()));
    }
    CK(ctx->ef2.ensure(sizeof(double) * 3 * std::max(N, 1)));
    const bool mixed = ctx->prm.precision == DDC_PREC_MIXED;
    const int ch2 = mixed ? efield_chunks_f32(NC, N) : efield_chunks(NC, N);
    if (!ctx->zfar_on) CK(ctx->ef_scratch.ensure(sizeof(double) * 3 * ((size_t)ch2 * N + 1)));
    // in mixed precision the force-only field of zeta uses FP32 pair
    // arithmetic, with the grouped multipole far field for large molecules
    auto efield = mixed ? launch_efield_f32 : launch_efield;
    CK(cudaEventRecord(ctx->ev_fork, ctx->st));
    CK(cudaStreamWaitEvent(ctx->st2, ctx->ev_fork, 0));
    {
      StageScope sc(ctx, ST_EFIELD, ctx->st2);
      if (ctx->zfar_on)
        CK(launch_zeta_field_far(Launch{ctx->st2, &ctx->launches}, N, ctx->sph.as<double4>(),
                                 ctx->cavoff.as<int>(), ctx->ccav.as<double>(),
                                 ctx->zeta.as<double>(), ctx->zg, ctx->zg_pk.as<float4>(),
                                 ctx->zg_M.as<float2>(), ctx->zg_scr.as<double>(),
                                 ctx->ef2.as<double>()));
      else
        CK(efield(Launch{ctx->st2, &ctx->launches}, NC, ctx->zeta.as<double>(),
                  ctx->ccav.as<double>(), N, ctx->csph.as<double>(), ctx->ef2.as<double>(),
                  ctx->ef_scratch.as<double>(), ch2, nullptr));
    }
    CK(cudaEventRecord(ctx->ev_join, ctx->st2));
    // forces and the zeta contraction on the main stream; whatever happens
    // there, the second stream is joined before this call returns, so no
    // later call can reuse ef2 / ef_scratch while the field is still running
    int frc = forces_dev(ctx, dphi, dsig, ds, dfx, true);
    if (frc == DDC_OK) {
      // solute field at the cavity (from the mkrhs pass) times zeta
      // (main.f90:241-253)
      StageScope sc(ctx, ST_CONTRACT);
      cudaError_t e = launch_zeta_efld_contract(ctx->L(), ctx->geo(), ctx->zeta.as<double>(),
                                                ctx->ef1.as<double>(), dfx);
      if (e != cudaSuccess) {
        cudaGetLastError();
        frc = fail(ctx, DDC_ERR_CUDA,
                   std::string("launch_zeta_efld_contract: ") + cudaGetErrorString(e));
      }
    }
    if (frc != DDC_OK) {
      cudaStreamSynchronize(ctx->st2);
      return frc;
    }
    // the field of zeta at the nuclei times the charges, after the join
    CK(cudaStreamWaitEvent(ctx->st, ctx->ev_join, 0));
    {
      StageScope sc(ctx, ST_CONTRACT);
      CK(launch_charge_efld_contract(ctx->L(), N, dq, ctx->ef2.as<double>(), dfx));
    }
    CKI(sync(ctx));
    const double t5 = now_s();
    inf->t_forces = t5 - t4;  // forces and both field contractions, overlapped
    inf->t_efld = 0.0;
  }
  CKI(finish_out(ctx, sigma, dsig, nv));
  if (ctx->prm.igrad) {
    CKI(finish_out(ctx, s, ds, nv));
    CKI(finish_out(ctx, fx, dfx, 3 * (size_t)N));
  }
  CKI(sync(ctx));
  inf->nsph = N;
  inf->ncav = NC;
  inf->nylm = ctx->nylm;
  inf->ngrid = ctx->ngrid;
  inf->ntriples = ctx->ntri;
  inf->npairs = ctx->npair;
  ctx->have_flow = true;
  return DDC_OK;
}


int ddc_batch_energy_forces(ddc_ctx* ctx, int nmol, const int* off, const double* charge,
                            const double* x, const double* y, const double* z,
                            const double* rvdw, double* esolv, double* fx, int* iters,
                            ddc_run_info* info) {
  if (!ctx || nmol <= 0 || !off || !esolv) return DDC_ERR_PARAM;
  cudaSetDevice(ctx->prm.device);
  if (off[0] != 0) return fail(ctx, DDC_ERR_PARAM, "off[0] must be 0");
  for (int k = 0; k < nmol; k++)
    if (off[k + 1] < off[k]) return fail(ctx, DDC_ERR_PARAM, "offsets must not decrease");
  const int N = off[nmol];
  ddc_run_info loc{};
  ddc_run_info* inf = info ? info : &loc;
  memset(inf, 0, sizeof(*inf));
  double t0 = now_s();
  // molecule partition: per-sphere index range of its molecule
  ctx->nmol = nmol;
  ctx->h_off.assign(off, off + nmol + 1);
  {
    std::vector<int2> mr(std::max(N, 1));
    for (int k = 0; k < nmol; k++)
      for (int i = off[k]; i < off[k + 1]; i++) mr[i] = make_int2(off[k], off[k + 1]);
    CK(ctx->mrange.ensure(sizeof(int2) * std::max(N, 1)));
    CK(cudaMemcpyAsync(ctx->mrange.p, mr.data(), sizeof(int2) * std::max(N, 1),
                       cudaMemcpyHostToDevice, ctx->st));
    CK(ctx->d_off.ensure(sizeof(int) * (nmol + 1)));
    CK(cudaMemcpyAsync(ctx->d_off.p, off, sizeof(int) * (nmol + 1), cudaMemcpyHostToDevice,
                       ctx->st));
  }
  ctx->batch_init = true;
  int rc = ddc_init(ctx, N, x, y, z, rvdw);
  ctx->batch_init = false;
  if (rc != DDC_OK) {
    ctx->nmol = 1;
    return rc;
  }
  ctx->nmol = nmol;
  double t1 = now_s();
  inf->t_init = t1 - t0;
  const int NC = ctx->ncav;
  const size_t nv = (size_t)N * ctx->nylm;
  CK(ctx->tr_cav.ensure(sizeof(int2) * std::max(NC, 1)));
  CK(ctx->tr_nuc.ensure(sizeof(int2) * std::max(N, 1)));
  CK(launch_batch_ranges(ctx->L(), N, ctx->ngrid, NC, ctx->mrange.as<int2>(), ctx->cavpt.as<int>(),
                         ctx->cavoff.as<int>(), ctx->tr_cav.as<int2>(), ctx->tr_nuc.as<int2>()));
  const double* dq;
  CKI(stage_in(ctx, charge, N, ctx->q, &dq));
  CK(ctx->phi.ensure(sizeof(double) * std::max(NC, 1)));
  double* dphi = ctx->phi.as<double>();
  double* dpsi = ctx->psi.as<double>();
  // the potential and (with forces) the solute field at the cavity, each
  // molecule's points from its own nuclei
  if (ctx->prm.igrad) CK(ctx->ef1.ensure(sizeof(double) * 3 * std::max(NC, 1)));
  CKI(solute_pot_field(ctx, dq, dphi, ctx->prm.igrad ? ctx->ef1.as<double>() : nullptr,
                       ctx->tr_cav.as<int2>()));
  CK(launch_psi(ctx->L(), N, ctx->nylm, dq, dpsi));
  CKI(sync(ctx));
  double t2 = now_s();
  inf->t_mkrhs = t2 - t1;
  double* dsig = ctx->sigma.as<double>();
  double* ds = ctx->s.as<double>();
  const long long n = (long long)nv;
  const bool paired = ctx->prm.igrad && ctx->prm.pair_solves;
  // direct solve (and the adjoint with it when paired)
  {
    double* rhs = ctx->rhs.as<double>();
    CK(ctx->gbuf.ensure(sizeof(double) * std::max<long long>((long long)N * ctx->ngrid, 1)));
    {
      StageScope sc(ctx, ST_RHS);
      CK(launch_wghpot(ctx->L(), ctx->geo(), dphi, ctx->gbuf.as<double>()));
      CK(launch_dgemm_nn(ctx->L(), ctx->nylm, N, ctx->ngrid, 1.0, ctx->bw.as<double>(),
                         ctx->nylm, ctx->gbuf.as<double>(), ctx->ngrid, rhs, ctx->nylm));
    }
    const bool learned = ctx->prm.guess == DDC_GUESS_LEARNED;
    if (learned)
      CKI(learned_guess(ctx, rhs, dpsi, dsig, ctx->prm.igrad ? ds : nullptr));
    else
      CK(launch_guess(ctx->L(), ctx->tb, n, rhs, dsig, ctx->prm.guess == DDC_GUESS_ZERO ? 1 : 0));
    std::vector<int> it(nmol), ita(nmol);
    BatchSys sys[2];
    CKI(batch_setup(ctx, sys[0], false, rhs, dsig, it.data(), &inf->direct, 0));
    if (paired) {
      // the adjoint right-hand side psi is known already: both systems share
      // each sweep's fused L / L* pass
      if (!learned)
        CK(launch_guess(ctx->L(), ctx->tb, n, dpsi, ds, ctx->prm.guess == DDC_GUESS_ZERO ? 1 : 0));
      CKI(batch_setup(ctx, sys[1], true, dpsi, ds, ita.data(), &inf->adjoint, 1));
    }
    if (ctx->prm.precision == DDC_PREC_MIXED)
      CKI(batch_run_mixed(ctx, sys, paired ? 2 : 1));
    else
      CKI(batch_run(ctx, sys, paired ? 2 : 1));
    if (iters)
      for (int k = 0; k < nmol; k++) {
        iters[2 * k] = it[k];
        if (paired) iters[2 * k + 1] = ita[k];
      }
  }
  CK(ctx->b_out.ensure(sizeof(double) * nmol));
  const double fep = 0.5 * ((ctx->prm.eps - 1.0) / ctx->prm.eps);
  CK(launch_batch_dot(ctx->L(), nmol, ctx->d_off.as<int>(), ctx->nylm, dsig, dpsi, fep,
                      ctx->b_out.as<double>()));
  CK(cudaMemcpyAsync(esolv, ctx->b_out.p, sizeof(double) * nmol, cudaMemcpyDeviceToHost, ctx->st));
  CKI(sync(ctx));
  double t3 = now_s();
  inf->t_direct = t3 - t2;
  if (ctx->prm.igrad) {
    if (!paired) {
      if (ctx->prm.guess != DDC_GUESS_LEARNED)
        CK(launch_guess(ctx->L(), ctx->tb, n, dpsi, ds, ctx->prm.guess == DDC_GUESS_ZERO ? 1 : 0));
      std::vector<int> it(nmol);
      BatchSys sys;
      CKI(batch_setup(ctx, sys, true, dpsi, ds, it.data(), &inf->adjoint, 0));
      if (ctx->prm.precision == DDC_PREC_MIXED)
        CKI(batch_run_mixed(ctx, &sys, 1));
      else
        CKI(batch_run(ctx, &sys, 1));
      if (iters)
        for (int k = 0; k < nmol; k++) iters[2 * k + 1] = it[k];
    }
    double t4 = now_s();
    inf->t_adjoint = t4 - t3;
    CK(ctx->fx.ensure(sizeof(double) * 3 * std::max(N, 1)));
    double* dfx = ctx->fx.as<double>();
    CKI(forces_dev(ctx, dphi, dsig, ds, dfx));
    CK(ctx->zeta.ensure(sizeof(double) * std::max(NC, 1)));
    {
      StageScope sc(ctx, ST_ZETA);
      CK(launch_mkxi(ctx->L(), ctx->tb, ctx->geo(), ctx->xig.as<double>(), fep,
                     ctx->zeta.as<double>()));
    }
    CKI(sync(ctx));
    double t5 = now_s();
    inf->t_forces = t5 - t4;
    CK(ctx->ef2.ensure(sizeof(double) * 3 * std::max(N, 1)));
    CK(ctx->ef_scratch.ensure(sizeof(double) * 3 * std::max((size_t)NC, (size_t)N)));
    {
      StageScope sc(ctx, ST_EFIELD);
      // each nucleus from the cavity points of its own molecule; in mixed
      // precision with FP32 pair arithmetic (FP64 sums), as the
      // single-molecule flow does for this force-only field
      auto efield = ctx->prm.precision == DDC_PREC_MIXED ? launch_efield_f32 : launch_efield;
      CK(efield(ctx->L(), NC, ctx->zeta.as<double>(), ctx->ccav.as<double>(), N,
                ctx->csph.as<double>(), ctx->ef2.as<double>(), ctx->ef_scratch.as<double>(), 1,
                ctx->tr_nuc.as<int2>()));
    }
    {
      StageScope sc(ctx, ST_CONTRACT);
      CK(launch_zeta_efld_contract(ctx->L(), ctx->geo(), ctx->zeta.as<double>(),
                                   ctx->ef1.as<double>(), dfx));
      CK(launch_charge_efld_contract(ctx->L(), N, dq, ctx->ef2.as<double>(), dfx));
    }
    CKI(finish_out(ctx, fx, dfx, 3 * (size_t)N));
    CKI(sync(ctx));
    inf->t_efld = now_s() - t5;
  }
  inf->nsph = N;
  inf->ncav = NC;
  inf->nylm = ctx->nylm;
  inf->ngrid = ctx->ngrid;
  inf->ntriples = ctx->ntri;
  inf->npairs = ctx->npair;
  ctx->have_flow = true;
  return DDC_OK;
}

// training rows of the learned guess from the last flow (ddc_guess.cu)
int ddc_guess_features(ddc_ctx* ctx, float* feat) {
  if (!ctx || !feat) return DDC_ERR_PARAM;
  if (!ctx->have_flow)
    return fail(ctx, DDC_ERR_STATE, "guess features need a ddc_energy_forces or batch call first");
  if (!ctx->gmodel) return fail(ctx, DDC_ERR_STATE, "no guess model (ddc_set_guess_model)");
  cudaSetDevice(ctx->prm.device);
  CK(launch_guess_features(ctx->L(), ctx->nsph, ctx->nylm, guess_nfeat(ctx->gmodel),
                           ctx->rhs.as<double>(), ctx->psi.as<double>(), ctx->sph.as<double4>(),
                           ctx->mrange_ptr(), feat));
  return sync(ctx);
}
int ddc_guess_targets(ddc_ctx* ctx, float* target) {
  if (!ctx || !target) return DDC_ERR_PARAM;
  if (!ctx->have_flow || !ctx->prm.igrad)
    return fail(ctx, DDC_ERR_STATE, "guess targets need an energy+force call (igrad=1) first");
  if (!ctx->gmodel) return fail(ctx, DDC_ERR_STATE, "no guess model (ddc_set_guess_model)");
  cudaSetDevice(ctx->prm.device);
  CK(launch_guess_targets(ctx->L(), ctx->tb, ctx->nsph, guess_nout(ctx->gmodel),
                          ctx->rhs.as<double>(), ctx->psi.as<double>(), ctx->sigma.as<double>(),
                          ctx->s.as<double>(), target));
  return sync(ctx);
}
int ddc_set_guess_model(ddc_ctx* ctx, ddc_guess* m) {
  if (!ctx) return DDC_ERR_PARAM;
  if (m && guess_lmax(m) != ctx->prm.lmax)
    return fail(ctx, DDC_ERR_PARAM, "guess model was built for another lmax");
  ctx->gmodel = m;
  return DDC_OK;
}

}  // extern "C"
