/*
 * ddc_ref.c -- CPU FP64 restatement of the reference ddCOSMO algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA library is
 * checked against, and the CPU baseline that bench.py times.  Nothing in the
 * product (ddpcm_b200/) links, loads or calls it.
 *
 * It restates, loop by loop and in the same summation order, the routines of
 * the Fortran reference (filippolipparini/ddPCM):
 *   ddinit        ddcosmo.f90:159-483      fsw/dfsw     ddcosmo.f90:566-655
 *   intrhs        ddcosmo.f90:789-821      ylmbas       ddcosmo.f90:830-895
 *   dbasis        ddcosmo.f90:904-1043     polleg       ddcosmo.f90:1056-1094
 *   trgev         ddcosmo.f90:1103-1125    intmlp       ddcosmo.f90:1140-1178
 *   wghpot        ddcosmo.f90:1187-1224    hsnorm       ddcosmo.f90:1233-1271
 *   adjrhs        ddcosmo.f90:1301-1384    fdoka        ddcosmo.f90:1436-1504
 *   fdokb         ddcosmo.f90:1511-1607    fdoga        ddcosmo.f90:1614-1650
 *   calcv         ddcosmo.f90:1671-1746    ddmkxi/zeta  ddcosmo.f90:1758-1806
 *   lx/lstarx/ldm1x/hnorm  matvec.f90:94-323
 *   jacobi_diis/diis/makeb/gjinv/rmsvec   jacobi_diis.f90:1-439 (loop at 102-176)
 *   cosmo         cosmo.f90:1-226          forces_dd    forces_dd.f90:91-164
 *   mkrhs         mkrhs.f90:86-123         efld         efld.f90:81-116
 *   main driver   main.f90:129-265 (units, order of force contractions)
 *   llgrid/gen_oh llgnew.f:5-681 (orbit parameters from lebedev_orbits.inc)
 *
 * Arrays use the reference's column-major shapes: X(nylm,nsph) is
 * X[isph*nylm + lm], grid(3,ngrid) is grid[3*ig + k], ui(ngrid,nsph) is
 * ui[isph*ngrid + ig].  Indices are 0-based internally.
 *
 * Parity status: the restatement is pinned against the printed intermediates
 * and results of the reference's regression logs (tests/NAME.log); no Fortran
 * compiler exists where it was written, so the reference itself was not run.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../ddpcm_b200/csrc/lebedev_orbits.inc"

#define NDIIS 25
#define NNGMAX_UNUSED 100

typedef struct {
  /* control parameters (ddcosmo.f90:106-107) */
  int lmax, ngrid, iconv, igrad, iprint, nthreads;
  double eps, eta;
  /* sizes */
  int nsph, ncav, nylm;
  /* geometry and tables */
  double *csph, *rsph, *w, *grid, *basis, *fact, *facl, *facs;
  int *inl, *nl; /* 0-based CSR */
  double *fi, *ui, *zi, *ccav;
  double pi, sq2;
  /* solver log of the last cosmo call */
  int last_iters;
  double last_norms[1024];
} ref_ctx;

/* ------------------------------------------------------------------ */
/* Lebedev grid: orbit expansion (gen_oh, llgnew.f:93-681)              */
/* ------------------------------------------------------------------ */
static int ref_gen_oh(int code, double a, double b, double v, double *x,
                      double *y, double *z, double *wt) {
  int n = 0;
#define P(X_, Y_, Z_) \
  do {                \
    x[n] = (X_);      \
    y[n] = (Y_);      \
    z[n] = (Z_);      \
    wt[n] = v;        \
    n++;              \
  } while (0)
  double c;
  switch (code) {
    case 1:
      a = 1.0;
      P(a, 0, 0); P(-a, 0, 0); P(0, a, 0); P(0, -a, 0); P(0, 0, a); P(0, 0, -a);
      break;
    case 2:
      a = sqrt(0.5);
      P(0, a, a); P(0, -a, a); P(0, a, -a); P(0, -a, -a);
      P(a, 0, a); P(-a, 0, a); P(a, 0, -a); P(-a, 0, -a);
      P(a, a, 0); P(-a, a, 0); P(a, -a, 0); P(-a, -a, 0);
      break;
    case 3:
      a = sqrt(1.0 / 3.0);
      P(a, a, a); P(-a, a, a); P(a, -a, a); P(-a, -a, a);
      P(a, a, -a); P(-a, a, -a); P(a, -a, -a); P(-a, -a, -a);
      break;
    case 4:
      b = sqrt(1.0 - 2.0 * a * a);
      P(a, a, b); P(-a, a, b); P(a, -a, b); P(-a, -a, b);
      P(a, a, -b); P(-a, a, -b); P(a, -a, -b); P(-a, -a, -b);
      P(a, b, a); P(-a, b, a); P(a, -b, a); P(-a, -b, a);
      P(a, b, -a); P(-a, b, -a); P(a, -b, -a); P(-a, -b, -a);
      P(b, a, a); P(-b, a, a); P(b, -a, a); P(-b, -a, a);
      P(b, a, -a); P(-b, a, -a); P(b, -a, -a); P(-b, -a, -a);
      break;
    case 5:
      b = sqrt(1.0 - a * a);
      P(a, b, 0); P(-a, b, 0); P(a, -b, 0); P(-a, -b, 0);
      P(b, a, 0); P(-b, a, 0); P(b, -a, 0); P(-b, -a, 0);
      P(a, 0, b); P(-a, 0, b); P(a, 0, -b); P(-a, 0, -b);
      P(b, 0, a); P(-b, 0, a); P(b, 0, -a); P(-b, 0, -a);
      P(0, a, b); P(0, -a, b); P(0, a, -b); P(0, -a, -b);
      P(0, b, a); P(0, -b, a); P(0, b, -a); P(0, -b, -a);
      break;
    case 6:
      c = sqrt(1.0 - a * a - b * b);
      P(a, b, c); P(-a, b, c); P(a, -b, c); P(-a, -b, c);
      P(a, b, -c); P(-a, b, -c); P(a, -b, -c); P(-a, -b, -c);
      P(a, c, b); P(-a, c, b); P(a, -c, b); P(-a, -c, b);
      P(a, c, -b); P(-a, c, -b); P(a, -c, -b); P(-a, -c, -b);
      P(b, a, c); P(-b, a, c); P(b, -a, c); P(-b, -a, c);
      P(b, a, -c); P(-b, a, -c); P(b, -a, -c); P(-b, -a, -c);
      P(b, c, a); P(-b, c, a); P(b, -c, a); P(-b, -c, a);
      P(b, c, -a); P(-b, c, -a); P(b, -c, -a); P(-b, -c, -a);
      P(c, a, b); P(-c, a, b); P(c, -a, b); P(-c, -a, b);
      P(c, a, -b); P(-c, a, -b); P(c, -a, -b); P(-c, -a, -b);
      P(c, b, a); P(-c, b, a); P(c, -b, a); P(-c, -b, a);
      P(c, b, -a); P(-c, b, -a); P(c, -b, -a); P(-c, -b, -a);
      break;
    default:
      return -1;
  }
#undef P
  return n;
}

/* Snap to the nearest Lebedev size; ties go to the smaller (ddcosmo.f90:188-199). */
int ref_snap_ngrid(int ngrid) {
  int best = 0, inear = 100000;
  for (int i = 0; i < LEB_NSIZES; i++) {
    int d = abs(leb_sizes[i] - ngrid);
    if (d < inear) {
      inear = d;
      best = i;
    }
  }
  return leb_sizes[best];
}

/* llgrid (llgnew.f:5-91): points and 4*pi-scaled weights. */
int ref_llgrid(int ngrid, double *w, double *grid) {
  int gi = -1;
  for (int i = 0; i < LEB_NSIZES; i++)
    if (leb_sizes[i] == ngrid) gi = i;
  if (gi < 0) return -1;
  double *x = malloc(sizeof(double) * ngrid * 4);
  double *y = x + ngrid, *z = y + ngrid, *wt = z + ngrid;
  int n = 0;
  for (int o = 0; o < leb_orbit_cnt[gi]; o++) {
    const struct leb_orbit_rec *r = &leb_orbits[leb_orbit_off[gi] + o];
    n += ref_gen_oh(r->code, r->a, r->b, r->v, x + n, y + n, z + n, wt + n);
  }
  double pi = 4.0 * atan(1.0);
  for (int i = 0; i < ngrid; i++) {
    w[i] = wt[i] * 4.0 * pi;
    grid[3 * i + 0] = x[i];
    grid[3 * i + 1] = y[i];
    grid[3 * i + 2] = z[i];
  }
  free(x);
  return n == ngrid ? 0 : -2;
}

/* ------------------------------------------------------------------ */
/* switch function and its derivative (ddcosmo.f90:566-655), se = -1    */
/* ------------------------------------------------------------------ */
static double eta5(double eta) {
  double e2 = eta * eta;
  return e2 * e2 * eta;
}

double ref_fsw(double t, double eta) {
  const double se = -1.0;
  double x = t - (se + 1.0) * eta / 2.0;
  double flow = 1.0 - eta;
  if (x >= 1.0) return 0.0;
  if (x <= flow) return 1.0;
  double a = 15.0 * eta - 12.0;
  double b = 10.0 * eta * eta - 15.0 * eta + 6.0;
  return ((x - 1.0) * (x - 1.0) * (1.0 - x) * (6.0 * x * x + a * x + b)) / eta5(eta);
}

double ref_dfsw(double t, double eta) {
  const double se = -1.0;
  double x = t - (se + 1.0) * eta / 2.0;
  double flow = 1.0 - eta;
  if (x >= 1.0) return 0.0;
  if (x <= flow) return 0.0;
  return 30.0 * (1.0 - x) * (x - 1.0) * (x - 1.0 + eta) * (x - 1.0 + eta) / eta5(eta);
}

/* ------------------------------------------------------------------ */
/* spherical harmonics                                                 */
/* ------------------------------------------------------------------ */
/* trgev (ddcosmo.f90:1103-1125): cos(m phi), sin(m phi) by Chebyshev. */
static void trgev(int lmax, double x, double y, double *cx, double *sx) {
  cx[0] = 1.0;
  sx[0] = 0.0;
  cx[1] = x;
  sx[1] = y;
  for (int m = 2; m <= lmax; m++) {
    cx[m] = 2.0 * x * cx[m - 1] - cx[m - 2];
    sx[m] = 2.0 * x * sx[m - 1] - sx[m - 2];
  }
}

/* polleg (ddcosmo.f90:1056-1094): associated Legendre P_l^m, no CS phase. */
static void polleg(int lmax, double x, double y, double *plm) {
  double fact = 1.0, pmm = 1.0, somx2 = y;
  for (int m = 0; m <= lmax; m++) {
    int ind = (m + 1) * (m + 1) - 1;
    plm[ind] = pmm;
    if (m == lmax) return;
    double fm = (double)m;
    double pmm1 = x * (2.0 * fm + 1.0) * pmm;
    int ind2 = ind + 2 * m + 2;
    plm[ind2] = pmm1;
    double pmmo = pmm;
    for (int l = m + 2; l <= lmax; l++) {
      double fl = (double)l;
      double pll = (x * (2.0 * fl - 1.0) * pmm1 - (fl + fm - 1.0) * pmm) / (fl - fm);
      int i2 = l * l + l;
      plm[i2 + m] = pll;
      pmm = pmm1;
      pmm1 = pll;
    }
    pmm = -pmmo * fact * somx2;
    fact = fact + 2.0;
  }
}

/* ylmbas (ddcosmo.f90:830-895).  vcos/vsin need max(lmax+1,2) entries. */
static void ylmbas(const ref_ctx *c, const double *x, double *basloc, double *vplm,
                   double *vcos, double *vsin) {
  int lmax = c->lmax;
  double cthe = x[2];
  double sthe = sqrt(1.0 - cthe * cthe);
  double cphi, sphi;
  if (sthe != 0.0) {
    cphi = x[0] / sthe;
    sphi = x[1] / sthe;
    trgev(lmax, cphi, sphi, vcos, vsin);
  } else {
    for (int m = 0; m <= lmax; m++) {
      vcos[m] = 1.0;
      vsin[m] = 0.0;
    }
  }
  polleg(lmax, cthe, sthe, vplm);
  for (int l = 0; l <= lmax; l++) {
    int ind = l * l + l;
    basloc[ind] = c->facs[ind] * vplm[ind];
    for (int m = 1; m <= l; m++) {
      double plm = vplm[ind + m];
      basloc[ind + m] = c->facs[ind + m] * plm * vcos[m];
      basloc[ind - m] = c->facs[ind - m] * plm * vsin[m];
    }
  }
}

/* dbasis (ddcosmo.f90:904-1043): Y and its surface gradient; dbsloc(3,nylm). */
static void dbasis(const ref_ctx *c, const double *x, double *basloc, double *dbsloc,
                   double *vplm, double *vcos, double *vsin) {
  int lmax = c->lmax;
  double cthe = x[2];
  double sthe = sqrt(1.0 - cthe * cthe);
  double cphi, sphi, et[3], ep[3];
  if (sthe != 0.0) {
    cphi = x[0] / sthe;
    sphi = x[1] / sthe;
  } else {
    cphi = 1.0;
    sphi = 0.0;
  }
  et[0] = cthe * cphi;
  et[1] = cthe * sphi;
  et[2] = -sthe;
  if (sthe != 0.0) {
    ep[0] = -sphi / sthe;
    ep[1] = cphi / sthe;
    ep[2] = 0.0;
  } else {
    ep[0] = 0.0;
    ep[1] = 1.0;
    ep[2] = 0.0;
  }
  if (sthe != 0.0) {
    trgev(lmax, cphi, sphi, vcos, vsin);
  } else {
    for (int m = 0; m <= lmax; m++) {
      vcos[m] = 1.0;
      vsin[m] = 0.0;
    }
  }
  /* VC/VS are declared integer in the reference (ddcosmo.f90:912): the
   * assignment truncates, so VC = 0 and VS = (int)cthe. */
  double VC = 0.0;
  double VS = (double)(int)cthe;
  polleg(lmax, cthe, sthe, vplm);
  int nylm = c->nylm;
  for (int k = 0; k < nylm; k++) basloc[k] = 0.0;
  for (int k = 0; k < 3 * nylm; k++) dbsloc[k] = 0.0;
  for (int l = 0; l <= lmax; l++) {
    int ind = l * l + l;
    double fln = c->facs[ind];
    basloc[ind] = fln * vplm[ind];
    if (l > 0) {
      for (int k = 0; k < 3; k++) dbsloc[3 * ind + k] = fln * vplm[ind + 1] * et[k];
    } else {
      for (int k = 0; k < 3; k++) dbsloc[3 * ind + k] = 0.0;
    }
    for (int m = 1; m <= l; m++) {
      fln = c->facs[ind + m];
      double plm = fln * vplm[ind + m];
      double pp1 = 0.0;
      if (m < l) pp1 = -0.5 * vplm[ind + m + 1];
      double pm1 = 0.5 * ((double)(l + m) * (double)(l - m + 1) * vplm[ind + m - 1]);
      double pp = pp1 + pm1;
      basloc[ind + m] = plm * vcos[m];
      if (sthe != 0.0) {
        for (int k = 0; k < 3; k++)
          dbsloc[3 * (ind + m) + k] =
              -fln * pp * vcos[m] * et[k] - (double)m * plm * vsin[m] * ep[k];
      } else {
        for (int k = 0; k < 3; k++)
          dbsloc[3 * (ind + m) + k] = -fln * pp * vcos[m] * et[k] - fln * pp * ep[k] * VC;
      }
      basloc[ind - m] = plm * vsin[m];
      if (sthe != 0.0) {
        for (int k = 0; k < 3; k++)
          dbsloc[3 * (ind - m) + k] =
              -fln * pp * vsin[m] * et[k] + (double)m * plm * vcos[m] * ep[k];
      } else {
        for (int k = 0; k < 3; k++)
          dbsloc[3 * (ind - m) + k] = -fln * pp * vsin[m] * et[k] - fln * pp * ep[k] * VS;
      }
    }
  }
}

/* intmlp (ddcosmo.f90:1140-1178). */
static double intmlp(const ref_ctx *c, double t, const double *sigma, const double *basloc) {
  double tt = 1.0, ss = 0.0;
  for (int l = 0; l <= c->lmax; l++) {
    int ind = l * l + l;
    double fac = tt / c->facl[ind];
    double d = 0.0;
    for (int m = -l; m <= l; m++) d += basloc[ind + m] * sigma[ind + m];
    ss = ss + fac * d;
    tt = tt * t;
  }
  return ss;
}

/* intrhs (ddcosmo.f90:789-821). */
static void intrhs(const ref_ctx *c, const double *x, double *xlm) {
  int nylm = c->nylm;
  for (int k = 0; k < nylm; k++) xlm[k] = 0.0;
  for (int ig = 0; ig < c->ngrid; ig++) {
    const double *b = c->basis + (size_t)ig * nylm;
    double wx = c->w[ig];
    for (int k = 0; k < nylm; k++) xlm[k] = xlm[k] + b[k] * wx * x[ig];
  }
}

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */
ref_ctx *ref_create(int lmax, int ngrid, int iconv, int igrad, double eps, double eta,
                    int nthreads) {
  ref_ctx *c = calloc(1, sizeof(ref_ctx));
  c->lmax = lmax;
  c->ngrid = ngrid;
  c->iconv = iconv;
  c->igrad = igrad;
  c->eps = eps;
  c->eta = eta;
  c->nthreads = nthreads;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  return c;
}

static void ref_free_arrays(ref_ctx *c) {
  free(c->csph); free(c->rsph); free(c->w); free(c->grid); free(c->basis);
  free(c->fact); free(c->facl); free(c->facs); free(c->inl); free(c->nl);
  free(c->fi); free(c->ui); free(c->zi); free(c->ccav);
  c->csph = c->rsph = c->w = c->grid = c->basis = c->fact = c->facl = c->facs = NULL;
  c->fi = c->ui = c->zi = c->ccav = NULL;
  c->inl = c->nl = NULL;
}

void ref_destroy(ref_ctx *c) {
  if (!c) return;
  ref_free_arrays(c);
  free(c);
}

/* ddinit (ddcosmo.f90:159-483); coordinates and radii in bohr. */
int ref_init(ref_ctx *c, int n, const double *x, const double *y, const double *z,
             const double *rvdw) {
  ref_free_arrays(c);
  c->pi = 4.0 * atan(1.0);
  c->sq2 = sqrt(2.0);
  c->nsph = n;
  c->ngrid = ref_snap_ngrid(c->ngrid);
  int lmax = c->lmax, ngrid = c->ngrid, nsph = n;
  int grad = c->igrad != 0;
  int nylm = (lmax + 1) * (lmax + 1);
  c->nylm = nylm;
  c->rsph = malloc(sizeof(double) * nsph);
  c->csph = malloc(sizeof(double) * 3 * nsph);
  c->w = malloc(sizeof(double) * ngrid);
  c->grid = malloc(sizeof(double) * 3 * ngrid);
  c->basis = malloc(sizeof(double) * (size_t)nylm * ngrid);
  c->inl = malloc(sizeof(int) * (nsph + 1));
  c->fi = calloc((size_t)ngrid * nsph, sizeof(double));
  c->ui = calloc((size_t)ngrid * nsph, sizeof(double));
  int nfact = 2 * lmax + 1 > 2 ? 2 * lmax + 1 : 2;
  c->fact = malloc(sizeof(double) * nfact);
  c->facl = malloc(sizeof(double) * nylm);
  c->facs = malloc(sizeof(double) * nylm);
  if (grad) c->zi = calloc((size_t)3 * ngrid * nsph, sizeof(double));

  /* factorials and normalisation (ddcosmo.f90:225-243) */
  c->fact[0] = 1.0;
  c->fact[1] = 1.0;
  for (int i = 3; i <= 2 * lmax + 1; i++) c->fact[i - 1] = (double)(i - 1) * c->fact[i - 2];
  for (int l = 0; l <= lmax; l++) {
    int ind = l * l + l;
    double fl = (2.0 * (double)l + 1.0) / (4.0 * c->pi);
    double ffl = sqrt(fl);
    for (int k = ind - l; k <= ind + l; k++) c->facl[k] = fl;
    c->facs[ind] = ffl;
    for (int m = 1; m <= l; m++) {
      double fnorm = c->sq2 * ffl * sqrt(c->fact[l - m] / c->fact[l + m]);
      if (m % 2 == 1) fnorm = -fnorm;
      c->facs[ind + m] = fnorm;
      c->facs[ind - m] = fnorm;
    }
  }
  for (int i = 0; i < nsph; i++) {
    c->csph[3 * i + 0] = x[i];
    c->csph[3 * i + 1] = y[i];
    c->csph[3 * i + 2] = z[i];
    c->rsph[i] = rvdw[i];
  }
  if (ref_llgrid(ngrid, c->w, c->grid) != 0) return -1;

  /* basis of spherical harmonics at the grid points (ddcosmo.f90:263-267) */
  int nv = lmax + 1 > 2 ? lmax + 1 : 2;
#pragma omp parallel
  {
    double *vplm = malloc(sizeof(double) * nylm);
    double *vc = malloc(sizeof(double) * nv), *vs = malloc(sizeof(double) * nv);
#pragma omp for
    for (int i = 0; i < ngrid; i++)
      ylmbas(c, c->grid + 3 * i, c->basis + (size_t)i * nylm, vplm, vc, vs);
    free(vplm); free(vc); free(vs);
  }

  /* CSR neighbour list, O(N^2) scan in index order (ddcosmo.f90:308-324) */
  size_t cap = (size_t)nsph * 16 + 16, lnl = 0;
  c->nl = malloc(sizeof(int) * cap);
  for (int i = 0; i < nsph; i++) {
    c->inl[i] = (int)lnl;
    for (int j = 0; j < nsph; j++) {
      if (i == j) continue;
      double dx = c->csph[3 * i] - c->csph[3 * j];
      double dy = c->csph[3 * i + 1] - c->csph[3 * j + 1];
      double dz = c->csph[3 * i + 2] - c->csph[3 * j + 2];
      double d2 = dx * dx + dy * dy + dz * dz;
      double r2 = (c->rsph[i] + c->rsph[j]) * (c->rsph[i] + c->rsph[j]);
      if (d2 <= r2) {
        if (lnl == cap) {
          cap *= 2;
          c->nl = realloc(c->nl, sizeof(int) * cap);
        }
        c->nl[lnl++] = j;
      }
    }
  }
  c->inl[nsph] = (int)lnl;

  /* fi, ui, zi (ddcosmo.f90:363-411) */
  double eta = c->eta;
#pragma omp parallel for schedule(static)
  for (int isph = 0; isph < nsph; isph++) {
    for (int i = 0; i < ngrid; i++) {
      double fi = 0.0;
      double zx = 0.0, zy = 0.0, zz = 0.0;
      for (int ii = c->inl[isph]; ii < c->inl[isph + 1]; ii++) {
        int jsph = c->nl[ii];
        double v[3];
        for (int k = 0; k < 3; k++)
          v[k] = c->csph[3 * isph + k] + c->rsph[isph] * c->grid[3 * i + k] - c->csph[3 * jsph + k];
        double vv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        double t = vv / c->rsph[jsph];
        double xt = ref_fsw(t, eta);
        double swthr = 1.0; /* 1 + (se+1)*eta/2 with se = -1 */
        if (grad && (t < swthr && t > swthr - eta)) {
          double fac = ref_dfsw(t, eta) / c->rsph[jsph];
          zx = zx + fac * v[0] / vv;
          zy = zy + fac * v[1] / vv;
          zz = zz + fac * v[2] / vv;
        }
        fi = fi + xt;
      }
      size_t p = (size_t)isph * ngrid + i;
      c->fi[p] = fi;
      c->ui[p] = fi <= 1.0 ? 1.0 - fi : 0.0;
      if (grad) {
        c->zi[3 * p + 0] = zx;
        c->zi[3 * p + 1] = zy;
        c->zi[3 * p + 2] = zz;
      }
    }
  }

  /* cavity points (ddcosmo.f90:422-468) */
  int ncav = 0;
  for (size_t p = 0; p < (size_t)nsph * ngrid; p++)
    if (c->ui[p] > 0.0) ncav++;
  c->ncav = ncav;
  c->ccav = malloc(sizeof(double) * 3 * (ncav > 0 ? ncav : 1));
  int ii = 0;
  for (int isph = 0; isph < nsph; isph++)
    for (int i = 0; i < ngrid; i++)
      if (c->ui[(size_t)isph * ngrid + i] > 0.0) {
        for (int k = 0; k < 3; k++)
          c->ccav[3 * ii + k] = c->csph[3 * isph + k] + c->rsph[isph] * c->grid[3 * i + k];
        ii++;
      }
  return 0;
}

/* ------------------------------------------------------------------ */
/* accessors                                                            */
/* ------------------------------------------------------------------ */
void ref_sizes(const ref_ctx *c, int *out) {
  out[0] = c->nsph;
  out[1] = c->ncav;
  out[2] = c->nylm;
  out[3] = c->ngrid;
  out[4] = c->nsph ? c->inl[c->nsph] : 0;
}

/* name: grid, w, basis, facs, facl, fi, ui, zi, ccav, csph, rsph */
int ref_get(const ref_ctx *c, const char *name, double *out) {
  size_t n = 0;
  const double *src = NULL;
  if (!strcmp(name, "grid")) { src = c->grid; n = 3 * (size_t)c->ngrid; }
  else if (!strcmp(name, "w")) { src = c->w; n = c->ngrid; }
  else if (!strcmp(name, "basis")) { src = c->basis; n = (size_t)c->nylm * c->ngrid; }
  else if (!strcmp(name, "facs")) { src = c->facs; n = c->nylm; }
  else if (!strcmp(name, "facl")) { src = c->facl; n = c->nylm; }
  else if (!strcmp(name, "fi")) { src = c->fi; n = (size_t)c->ngrid * c->nsph; }
  else if (!strcmp(name, "ui")) { src = c->ui; n = (size_t)c->ngrid * c->nsph; }
  else if (!strcmp(name, "zi")) { src = c->zi; n = src ? 3 * (size_t)c->ngrid * c->nsph : 0; }
  else if (!strcmp(name, "ccav")) { src = c->ccav; n = 3 * (size_t)c->ncav; }
  else if (!strcmp(name, "csph")) { src = c->csph; n = 3 * (size_t)c->nsph; }
  else if (!strcmp(name, "rsph")) { src = c->rsph; n = c->nsph; }
  else return -1;
  if (src && n) memcpy(out, src, n * sizeof(double));
  return (int)n;
}

void ref_get_csr(const ref_ctx *c, int *inl, int *nl) {
  memcpy(inl, c->inl, sizeof(int) * (c->nsph + 1));
  memcpy(nl, c->nl, sizeof(int) * c->inl[c->nsph]);
}

/* ------------------------------------------------------------------ */
/* operators (matvec.f90)                                               */
/* ------------------------------------------------------------------ */
/* calcv (ddcosmo.f90:1671-1746) for one sphere. */
static void calcv(const ref_ctx *c, int isph, double *pot, const double *sigma, double *basloc,
                  double *vplm, double *vcos, double *vsin) {
  int ngrid = c->ngrid, nylm = c->nylm;
  double eta = c->eta;
  for (int its = 0; its < ngrid; its++) pot[its] = 0.0;
  for (int its = 0; its < ngrid; its++) {
    size_t p = (size_t)isph * ngrid + its;
    if (c->ui[p] < 1.0) {
      for (int ij = c->inl[isph]; ij < c->inl[isph + 1]; ij++) {
        int jsph = c->nl[ij];
        double vij[3];
        for (int k = 0; k < 3; k++)
          vij[k] = c->csph[3 * isph + k] + c->rsph[isph] * c->grid[3 * its + k] - c->csph[3 * jsph + k];
        double vvij = sqrt(vij[0] * vij[0] + vij[1] * vij[1] + vij[2] * vij[2]);
        double tij = vvij / c->rsph[jsph];
        if (tij < 1.0) {
          double sij[3] = {vij[0] / vvij, vij[1] / vvij, vij[2] / vvij};
          double xij = ref_fsw(tij, eta);
          double oij = c->fi[p] > 1.0 ? xij / c->fi[p] : xij;
          ylmbas(c, sij, basloc, vplm, vcos, vsin);
          pot[its] = pot[its] + oij * intmlp(c, tij, sigma + (size_t)jsph * nylm, basloc);
        }
      }
    }
  }
}

/* lx (matvec.f90:94-148): y = off-diagonal L x. */
void ref_lx(const ref_ctx *c, const double *x, double *y) {
  int nylm = c->nylm, nv = c->lmax + 1 > 2 ? c->lmax + 1 : 2;
#pragma omp parallel
  {
    double *pot = malloc(sizeof(double) * c->ngrid);
    double *basloc = malloc(sizeof(double) * nylm), *vplm = malloc(sizeof(double) * nylm);
    double *vc = malloc(sizeof(double) * nv), *vs = malloc(sizeof(double) * nv);
#pragma omp for schedule(dynamic)
    for (int isph = 0; isph < c->nsph; isph++) {
      calcv(c, isph, pot, x, basloc, vplm, vc, vs);
      double *yi = y + (size_t)isph * nylm;
      intrhs(c, pot, yi);
      for (int k = 0; k < nylm; k++) yi[k] = -yi[k];
    }
    free(pot); free(basloc); free(vplm); free(vc); free(vs);
  }
}

/* adjrhs (ddcosmo.f90:1301-1384) for one sphere. */
static void adjrhs(const ref_ctx *c, int isph, const double *xi, double *vlm, double *basloc,
                   double *vplm, double *vcos, double *vsin) {
  int ngrid = c->ngrid;
  double eta = c->eta;
  for (int ij = c->inl[isph]; ij < c->inl[isph + 1]; ij++) {
    int jsph = c->nl[ij];
    for (int ig = 0; ig < ngrid; ig++) {
      double vji[3];
      for (int k = 0; k < 3; k++)
        vji[k] = c->csph[3 * jsph + k] + c->rsph[jsph] * c->grid[3 * ig + k] - c->csph[3 * isph + k];
      double vvji = sqrt(vji[0] * vji[0] + vji[1] * vji[1] + vji[2] * vji[2]);
      double tji = vvji / c->rsph[isph];
      if (tji < 1.0) {
        double sji[3] = {vji[0] / vvji, vji[1] / vvji, vji[2] / vvji};
        double xji = ref_fsw(tji, eta);
        size_t pj = (size_t)jsph * ngrid + ig;
        double oji = c->fi[pj] > 1.0 ? xji / c->fi[pj] : xji;
        ylmbas(c, sji, basloc, vplm, vcos, vsin);
        double t = 1.0;
        double fac = c->w[ig] * xi[pj] * oji;
        for (int l = 0; l <= c->lmax; l++) {
          int ind = l * l + l;
          double ffac = fac * t / c->facl[ind];
          for (int m = -l; m <= l; m++) vlm[ind + m] = vlm[ind + m] + ffac * basloc[ind + m];
          t = t * tji;
        }
      }
    }
  }
}

/* lstarx (matvec.f90:161-235): y = off-diagonal L* x. */
void ref_lstarx(const ref_ctx *c, const double *x, double *y) {
  int nylm = c->nylm, ngrid = c->ngrid, nv = c->lmax + 1 > 2 ? c->lmax + 1 : 2;
  double *xi = malloc(sizeof(double) * (size_t)ngrid * c->nsph);
#pragma omp parallel for
  for (int isph = 0; isph < c->nsph; isph++)
    for (int ig = 0; ig < ngrid; ig++) {
      double d = 0.0;
      for (int k = 0; k < nylm; k++) d += x[(size_t)isph * nylm + k] * c->basis[(size_t)ig * nylm + k];
      xi[(size_t)isph * ngrid + ig] = d;
    }
#pragma omp parallel
  {
    double *basloc = malloc(sizeof(double) * nylm), *vplm = malloc(sizeof(double) * nylm);
    double *vc = malloc(sizeof(double) * nv), *vs = malloc(sizeof(double) * nv);
#pragma omp for schedule(dynamic)
    for (int isph = 0; isph < c->nsph; isph++) {
      double *yi = y + (size_t)isph * nylm;
      for (int k = 0; k < nylm; k++) yi[k] = 0.0;
      adjrhs(c, isph, xi, yi, basloc, vplm, vc, vs);
      for (int k = 0; k < nylm; k++) yi[k] = -yi[k];
    }
    free(basloc); free(vplm); free(vc); free(vs);
  }
  free(xi);
}

/* ldm1x (matvec.f90:246-269). */
void ref_ldm1x(const ref_ctx *c, const double *x, double *y) {
  int nylm = c->nylm;
  for (int isph = 0; isph < c->nsph; isph++)
    for (int k = 0; k < nylm; k++) y[(size_t)isph * nylm + k] = c->facl[k] * x[(size_t)isph * nylm + k];
}

/* hsnorm (ddcosmo.f90:1233-1271). */
static double hsnorm(const ref_ctx *c, const double *u) {
  double un = 0.0;
  for (int l = 0; l <= c->lmax; l++) {
    int ind = l * l + l;
    double fac = 1.0 / (1.0 + (double)l);
    for (int m = -l; m <= l; m++) un = un + fac * u[ind + m] * u[ind + m];
  }
  return sqrt(un);
}

/* hnorm (matvec.f90:281-323) with rmsvec (jacobi_diis.f90:400-439). */
double ref_hnorm(const ref_ctx *c, const double *x) {
  double vrms = 0.0;
  for (int isph = 0; isph < c->nsph; isph++) {
    double u = hsnorm(c, x + (size_t)isph * c->nylm);
    vrms = vrms + u * u;
  }
  return sqrt(vrms / (double)c->nsph);
}

/* ------------------------------------------------------------------ */
/* Jacobi / DIIS (jacobi_diis.f90)                                      */
/* ------------------------------------------------------------------ */
#define B(j, k) b[((k)-1) * (NDIIS + 1) + ((j)-1)] /* 1-based column-major (ndiis+1)^2 */

static double dotv(size_t n, const double *a, const double *b) {
  double s = 0.0;
  for (size_t i = 0; i < n; i++) s = s + a[i] * b[i];
  return s;
}

/* gjinv: Gauss-Jordan with full pivoting, nrhs = 1 (jacobi_diis.f90:272-360). */
int ref_gjinv(int n, double *a, double *bv) {
#define A(j, k) a[((k)-1) * n + ((j)-1)]
  int *indxc = calloc(n + 1, sizeof(int)), *indxr = calloc(n + 1, sizeof(int));
  int *piv = calloc(n + 1, sizeof(int));
  double *scr = malloc(sizeof(double) * (n + 1));
  int ok = 0, irow = 0, icol = 0;
  for (int i = 1; i <= n; i++) {
    double big = 0.0;
    for (int j = 1; j <= n; j++)
      if (piv[j] != 1)
        for (int k = 1; k <= n; k++)
          if (piv[k] == 0)
            if (fabs(A(j, k)) > big) {
              big = fabs(A(j, k));
              irow = j;
              icol = k;
            }
    if (icol == 0) goto done; /* all-zero matrix: singular */
    piv[icol] += 1;
    if (piv[icol] > 1) goto done;
    if (irow != icol) {
      for (int k = 1; k <= n; k++) {
        double s = A(irow, k);
        A(irow, k) = A(icol, k);
        A(icol, k) = s;
      }
      double s = bv[irow - 1];
      bv[irow - 1] = bv[icol - 1];
      bv[icol - 1] = s;
    }
    indxr[i] = irow;
    indxc[i] = icol;
    if (A(icol, icol) == 0.0) goto done;
    double pinv = 1.0 / A(icol, icol);
    A(icol, icol) = 1.0;
    for (int k = 1; k <= n; k++) A(icol, k) = A(icol, k) * pinv;
    bv[icol - 1] = bv[icol - 1] * pinv;
    for (int j = 1; j <= n; j++)
      if (j != icol) {
        double dum = A(j, icol);
        A(j, icol) = 0.0;
        for (int k = 1; k <= n; k++) A(j, k) = A(j, k) - A(icol, k) * dum;
        bv[j - 1] = bv[j - 1] - bv[icol - 1] * dum;
      }
  }
  for (int j = n; j >= 1; j--)
    if (indxr[j] != indxc[j])
      for (int k = 1; k <= n; k++) {
        double s = A(k, indxr[j]);
        A(k, indxr[j]) = A(k, indxc[j]);
        A(k, indxc[j]) = s;
      }
  ok = 1;
done:
  free(indxc); free(indxr); free(piv); free(scr);
  return ok;
#undef A
}

/* diis (jacobi_diis.f90:183-230) and makeb (232-270). */
static void diis(size_t n, int *nmat, double *x, double *e, double *b, double *xnew) {
  if (*nmat >= NDIIS) {
    for (int j = 2; j <= *nmat - 10; j++)
      for (int k = 2; k <= *nmat - 10; k++) B(j, k) = B(j + 10, k + 10);
    for (int j = 1; j <= *nmat - 10; j++) {
      memcpy(x + (j - 1) * n, x + (j + 9) * n, n * sizeof(double));
      memcpy(e + (j - 1) * n, e + (j + 9) * n, n * sizeof(double));
    }
    *nmat -= 10;
  }
  int nm = *nmat, nmat1 = nm + 1;
  /* makeb */
  if (nm == 1) {
    B(1, 1) = 0.0;
    B(1, 2) = 1.0;
    B(2, 1) = 1.0;
    B(2, 2) = dotv(n, e, e);
  } else {
    B(nm + 1, 1) = 1.0;
    B(1, nm + 1) = 1.0;
    for (int i = 1; i <= nm - 1; i++) {
      double bij = dotv(n, e + (i - 1) * n, e + (nm - 1) * n);
      B(nm + 1, i + 1) = bij;
      B(i + 1, nm + 1) = bij;
    }
    B(nm + 1, nm + 1) = dotv(n, e + (nm - 1) * n, e + (nm - 1) * n);
  }
  double bloc[(NDIIS + 1) * (NDIIS + 1)], cex[NDIIS + 1];
  for (int k = 1; k <= nmat1; k++)
    for (int j = 1; j <= nmat1; j++) bloc[(k - 1) * nmat1 + (j - 1)] = B(j, k);
  for (int j = 0; j < nmat1; j++) cex[j] = 0.0;
  cex[0] = 1.0;
  if (!ref_gjinv(nmat1, bloc, cex)) {
    *nmat = 1;
    return;
  }
  for (size_t k = 0; k < n; k++) xnew[k] = 0.0;
  for (int i = 1; i <= nm; i++) {
    const double *xi = x + (i - 1) * n;
    double ci = cex[i];
    for (size_t k = 0; k < n; k++) xnew[k] = xnew[k] + ci * xi[k];
  }
  *nmat = nm + 1;
}

typedef void (*ref_matvec_fn)(const ref_ctx *, const double *, double *);

/* jacobi_diis (jacobi_diis.f90:1-176), norm mode 4 (hnorm), DIIS on. */
static int jacobi_diis(ref_ctx *c, size_t n, double tol, const double *rhs, double *x,
                       int n_iter, ref_matvec_fn matvec, double *norms) {
  double *xnew = malloc(sizeof(double) * n), *y = malloc(sizeof(double) * n);
  double *xd = malloc(sizeof(double) * n * NDIIS), *ed = malloc(sizeof(double) * n * NDIIS);
  double b[(NDIIS + 1) * (NDIIS + 1)];
  memset(b, 0, sizeof(b));
  int nmat = 1, it, ok = 0;
  for (it = 1; it <= n_iter; it++) {
    matvec(c, x, y);
    for (size_t k = 0; k < n; k++) y[k] = rhs[k] - y[k];
    ref_ldm1x(c, y, xnew);
    memcpy(xd + (nmat - 1) * n, xnew, n * sizeof(double));
    for (size_t k = 0; k < n; k++) ed[(nmat - 1) * n + k] = xnew[k] - x[k];
    diis(n, &nmat, xd, ed, b, xnew);
    for (size_t k = 0; k < n; k++) x[k] = xnew[k] - x[k];
    double rms = ref_hnorm(c, x);
    if (norms && it <= 1024) norms[it - 1] = rms;
    ok = rms < tol;
    memcpy(x, xnew, n * sizeof(double));
    if (ok) break;
  }
  free(xnew); free(y); free(xd); free(ed);
  c->last_iters = ok ? it : n_iter;
  return ok;
}

/* Timing sample of the solver's vector work (CPU baseline only): the
 * jacobi_diis loop above, run for `iters` iterations on a vector of the
 * context's size, with the operator replaced by a cheap shift (y_k = 0.3 x_{k+1},
 * which keeps the DIIS history non-degenerate) and a tolerance of zero so it
 * never stops early.  Everything else -- D^-1, the history copies, the Gram
 * row, the Gauss-Jordan solve, the extrapolation and the H-norm -- is the
 * reference's serial per-iteration work (jacobi_diis.f90:102-176, 183-270).
 * Returns the number of iterations run; *op_share is the fraction of them
 * spent in the stand-in operator, measured separately. */
static void shift_op(const ref_ctx *c, const double *x, double *y) {
  size_t n = (size_t)c->nylm * c->nsph;
  for (size_t k = 0; k + 1 < n; k++) y[k] = 0.3 * x[k + 1];
  y[n - 1] = 0.3 * x[0];
}
int ref_diis_sample(ref_ctx *c, int iters, double *seconds, double *op_seconds) {
  size_t n = (size_t)c->nylm * c->nsph;
  if (n == 0) return 0;
  double *rhs = malloc(sizeof(double) * n), *x = malloc(sizeof(double) * n);
  for (size_t k = 0; k < n; k++) {
    rhs[k] = 1.0 + 1e-3 * (double)(k % 97);
    x[k] = 0.0;
  }
#ifdef _OPENMP
  double t0 = omp_get_wtime();
#endif
  jacobi_diis(c, n, 0.0, rhs, x, iters, shift_op, NULL);
#ifdef _OPENMP
  double t1 = omp_get_wtime();
  for (int it = 0; it < iters; it++) shift_op(c, x, rhs);
  double t2 = omp_get_wtime();
  *seconds = t1 - t0;
  *op_seconds = t2 - t1;
#else
  *seconds = 0.0;
  *op_seconds = 0.0;
#endif
  free(rhs);
  free(x);
  return iters;
}

/* wghpot (ddcosmo.f90:1187-1224). */
static void wghpot(const ref_ctx *c, const double *phi, double *g) {
  int ic = 0;
  for (size_t p = 0; p < (size_t)c->nsph * c->ngrid; p++) {
    g[p] = 0.0;
    if (c->ui[p] != 0.0) {
      g[p] = -c->ui[p] * phi[ic];
      ic++;
    }
  }
}

/* cosmo (cosmo.f90:1-226).  Returns 0 on convergence, 1 otherwise (the
 * reference stops the program instead). iters/norms report the solver log. */
int ref_cosmo(ref_ctx *c, int star, int cart, const double *phi, const double *glm,
              const double *psi, double *sigma, double *esolv, int *iters, double *norms) {
  int nylm = c->nylm, nsph = c->nsph;
  size_t n = (size_t)nylm * nsph;
  double tol = pow(10.0, -(double)c->iconv);
  int n_iter = 200, ok;
  if (!star) {
    double *rhs = malloc(sizeof(double) * n);
    if (cart) {
      double *g = malloc(sizeof(double) * (size_t)c->ngrid * nsph);
      wghpot(c, phi, g);
#pragma omp parallel for
      for (int isph = 0; isph < nsph; isph++)
        intrhs(c, g + (size_t)isph * c->ngrid, rhs + (size_t)isph * nylm);
      free(g);
    } else {
      memcpy(rhs, glm, n * sizeof(double));
    }
    for (int isph = 0; isph < nsph; isph++)
      for (int k = 0; k < nylm; k++) sigma[(size_t)isph * nylm + k] = c->facl[k] * rhs[(size_t)isph * nylm + k];
    ok = jacobi_diis(c, n, tol, rhs, sigma, n_iter, ref_lx, norms);
    *esolv = 0.5 * ((c->eps - 1.0) / c->eps) * dotv(n, sigma, psi);
    free(rhs);
  } else {
    for (int isph = 0; isph < nsph; isph++)
      for (int k = 0; k < nylm; k++) sigma[(size_t)isph * nylm + k] = c->facl[k] * psi[(size_t)isph * nylm + k];
    ok = jacobi_diis(c, n, tol, psi, sigma, n_iter, ref_lstarx, norms);
  }
  if (iters) *iters = c->last_iters;
  return ok ? 0 : 1;
}

/* Expose the RHS assembly (wghpot + intrhs) on its own. */
void ref_rhs(const ref_ctx *c, const double *phi, double *rhs) {
  double *g = malloc(sizeof(double) * (size_t)c->ngrid * c->nsph);
  wghpot(c, phi, g);
  for (int isph = 0; isph < c->nsph; isph++)
    intrhs(c, g + (size_t)isph * c->ngrid, rhs + (size_t)isph * c->nylm);
  free(g);
}

/* ------------------------------------------------------------------ */
/* forces (ddcosmo.f90:1436-1650, forces_dd.f90:91-164)                 */
/* ------------------------------------------------------------------ */
typedef struct {
  double *basloc, *dbsloc, *vplm, *vcos, *vsin;
} ref_ws;

static void fdoka(const ref_ctx *c, int isph, const double *sigma, const double *xi_i, ref_ws *ws,
                  double *fx) {
  const double eta = c->eta, tlow = 1.0 - eta, thigh = 1.0;
  int ngrid = c->ngrid, nylm = c->nylm;
  for (int ig = 0; ig < ngrid; ig++) {
    double va[3] = {0, 0, 0};
    size_t p = (size_t)isph * ngrid + ig;
    for (int ij = c->inl[isph]; ij < c->inl[isph + 1]; ij++) {
      int jsph = c->nl[ij];
      double vij[3];
      for (int k = 0; k < 3; k++)
        vij[k] = c->csph[3 * isph + k] + c->rsph[isph] * c->grid[3 * ig + k] - c->csph[3 * jsph + k];
      double vvij = sqrt(vij[0] * vij[0] + vij[1] * vij[1] + vij[2] * vij[2]);
      double tij = vvij / c->rsph[jsph];
      if (tij >= thigh) continue;
      double sij[3] = {vij[0] / vvij, vij[1] / vvij, vij[2] / vvij};
      dbasis(c, sij, ws->basloc, ws->dbsloc, ws->vplm, ws->vcos, ws->vsin);
      double alp[3] = {0, 0, 0};
      double t = 1.0;
      const double *sj = sigma + (size_t)jsph * nylm;
      for (int l = 1; l <= c->lmax; l++) {
        int ind = l * l + l;
        double fl = (double)l;
        double fac = t / c->facl[ind];
        for (int m = -l; m <= l; m++) {
          double f2 = fac * sj[ind + m];
          double f1 = f2 * fl * ws->basloc[ind + m];
          for (int k = 0; k < 3; k++) alp[k] = alp[k] + f1 * sij[k] + f2 * ws->dbsloc[3 * (ind + m) + k];
        }
        t = t * tij;
      }
      double beta = intmlp(c, tij, sj, ws->basloc);
      double xij = ref_fsw(tij, eta), oij, f2;
      if (c->fi[p] > 1.0) {
        oij = xij / c->fi[p];
        f2 = -oij / c->fi[p];
      } else {
        oij = xij;
        f2 = 0.0;
      }
      double f1 = oij / c->rsph[jsph];
      for (int k = 0; k < 3; k++) va[k] = va[k] + f1 * alp[k] + beta * f2 * c->zi[3 * p + k];
      if (tij > tlow) {
        double f3 = beta * ref_dfsw(tij, eta) / c->rsph[jsph];
        if (c->fi[p] > 1.0) f3 = f3 / c->fi[p];
        for (int k = 0; k < 3; k++) va[k] = va[k] + f3 * sij[k];
      }
    }
    for (int k = 0; k < 3; k++) fx[k] = fx[k] - c->w[ig] * xi_i[ig] * va[k];
  }
}

static void fdokb(const ref_ctx *c, int isph, const double *sigma, const double *xi, ref_ws *ws,
                  double *fx) {
  const double eta = c->eta, tlow = 1.0 - eta, thigh = 1.0;
  int ngrid = c->ngrid, nylm = c->nylm;
  const double *si = sigma + (size_t)isph * nylm;
  for (int ig = 0; ig < ngrid; ig++) {
    double vb[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
    for (int ji = c->inl[isph]; ji < c->inl[isph + 1]; ji++) {
      int jsph = c->nl[ji];
      size_t pj = (size_t)jsph * ngrid + ig;
      double vji[3];
      for (int k = 0; k < 3; k++)
        vji[k] = c->csph[3 * jsph + k] + c->rsph[jsph] * c->grid[3 * ig + k] - c->csph[3 * isph + k];
      double vvji = sqrt(vji[0] * vji[0] + vji[1] * vji[1] + vji[2] * vji[2]);
      double tji = vvji / c->rsph[isph];
      if (tji > thigh) continue;
      double sji[3] = {vji[0] / vvji, vji[1] / vvji, vji[2] / vvji};
      dbasis(c, sji, ws->basloc, ws->dbsloc, ws->vplm, ws->vcos, ws->vsin);
      double alp[3] = {0, 0, 0};
      double t = 1.0;
      for (int l = 1; l <= c->lmax; l++) {
        int ind = l * l + l;
        double fl = (double)l;
        double fac = t / c->facl[ind];
        for (int m = -l; m <= l; m++) {
          double f2 = fac * si[ind + m];
          double f1 = f2 * fl * ws->basloc[ind + m];
          for (int k = 0; k < 3; k++) alp[k] = alp[k] + f1 * sji[k] + f2 * ws->dbsloc[3 * (ind + m) + k];
        }
        t = t * tji;
      }
      double xji = ref_fsw(tji, eta);
      double oji = c->fi[pj] > 1.0 ? xji / c->fi[pj] : xji;
      double f1 = oji / c->rsph[isph];
      for (int k = 0; k < 3; k++) vb[k] = vb[k] + f1 * alp[k] * xi[pj];
      if (tji > tlow) {
        double beta = intmlp(c, tji, si, ws->basloc);
        double di, fac;
        if (c->fi[pj] > 1.0) {
          di = 1.0 / c->fi[pj];
          fac = di * xji;
          int proc = 0;
          double bsum = 0.0;
          for (int jk = c->inl[jsph]; jk < c->inl[jsph + 1]; jk++) {
            int ksph = c->nl[jk];
            double vjk[3];
            for (int k = 0; k < 3; k++)
              vjk[k] = c->csph[3 * jsph + k] + c->rsph[jsph] * c->grid[3 * ig + k] - c->csph[3 * ksph + k];
            double vvjk = sqrt(vjk[0] * vjk[0] + vjk[1] * vjk[1] + vjk[2] * vjk[2]);
            double tjk = vvjk / c->rsph[ksph];
            if (ksph != isph && tjk <= thigh) {
              proc = 1;
              double sjk[3] = {vjk[0] / vvjk, vjk[1] / vvjk, vjk[2] / vvjk};
              ylmbas(c, sjk, ws->basloc, ws->vplm, ws->vcos, ws->vsin);
              double g1 = intmlp(c, tjk, sigma + (size_t)ksph * nylm, ws->basloc);
              double xjk = ref_fsw(tjk, eta);
              bsum = bsum + g1 * xjk;
            }
          }
          if (proc) {
            double g1 = di * di * ref_dfsw(tji, eta) / c->rsph[isph];
            double g2 = g1 * xi[pj] * bsum;
            for (int k = 0; k < 3; k++) vc[k] = vc[k] + g2 * sji[k];
          }
        } else {
          di = 1.0;
          fac = 0.0;
        }
        double f2 = (1.0 - fac) * di * ref_dfsw(tji, eta) / c->rsph[isph];
        for (int k = 0; k < 3; k++) vb[k] = vb[k] + f2 * xi[pj] * beta * sji[k];
      }
    }
    for (int k = 0; k < 3; k++) fx[k] = fx[k] + c->w[ig] * (vb[k] - vc[k]);
  }
}

static void fdoga(const ref_ctx *c, int isph, const double *xi, const double *phiexp, double *fx) {
  const double eta = c->eta;
  int ngrid = c->ngrid;
  for (int ig = 0; ig < ngrid; ig++) {
    double alp[3] = {0, 0, 0};
    size_t p = (size_t)isph * ngrid + ig;
    if (c->ui[p] > 0.0 && c->ui[p] < 1.0)
      for (int k = 0; k < 3; k++) alp[k] = alp[k] + phiexp[p] * xi[p] * c->zi[3 * p + k];
    for (int ji = c->inl[isph]; ji < c->inl[isph + 1]; ji++) {
      int jsph = c->nl[ji];
      size_t pj = (size_t)jsph * ngrid + ig;
      double vji[3];
      for (int k = 0; k < 3; k++)
        vji[k] = c->csph[3 * jsph + k] + c->rsph[jsph] * c->grid[3 * ig + k] - c->csph[3 * isph + k];
      double vvji = sqrt(vji[0] * vji[0] + vji[1] * vji[1] + vji[2] * vji[2]);
      double tji = vvji / c->rsph[isph];
      double swthr = 1.0;
      if (tji < swthr && tji > swthr - eta && c->ui[pj] > 0.0) {
        double sji[3] = {vji[0] / vvji, vji[1] / vvji, vji[2] / vvji};
        double fac = -ref_dfsw(tji, eta) / c->rsph[isph];
        for (int k = 0; k < 3; k++) alp[k] = alp[k] + fac * phiexp[pj] * xi[pj] * sji[k];
      }
    }
    for (int k = 0; k < 3; k++) fx[k] = fx[k] - c->w[ig] * alp[k];
  }
}

/* forces_dd (forces_dd.f90:91-164) restricted to the sphere ranges
 * [rg[2r], rg[2r+1]), r < nrg: those rows of fx(3,n) are overwritten (the
 * whole molecule, or a bounded timing sample). */
int ref_forces_dd_ranges(const ref_ctx *c, const double *phi, const double *sigma,
                         const double *s, double *fx, const int *rg, int nrg);
int ref_forces_dd(const ref_ctx *c, const double *phi, const double *sigma, const double *s,
                  double *fx) {
  int rg[2] = {0, c->nsph};
  return ref_forces_dd_ranges(c, phi, sigma, s, fx, rg, 1);
}
int ref_forces_dd_ranges(const ref_ctx *c, const double *phi, const double *sigma,
                         const double *s, double *fx, const int *rg, int nrg) {
  int nsph = c->nsph, ngrid = c->ngrid, nylm = c->nylm;
  if (!c->zi) return -1;
  double *xi = malloc(sizeof(double) * (size_t)ngrid * nsph);
  double *phiexp = calloc((size_t)ngrid * nsph, sizeof(double));
#pragma omp parallel for
  for (int isph = 0; isph < nsph; isph++)
    for (int ig = 0; ig < ngrid; ig++) {
      double d = 0.0;
      for (int k = 0; k < nylm; k++) d += s[(size_t)isph * nylm + k] * c->basis[(size_t)ig * nylm + k];
      xi[(size_t)isph * ngrid + ig] = d;
    }
  int ii = 0;
  for (size_t p = 0; p < (size_t)nsph * ngrid; p++)
    if (c->ui[p] > 0.0) phiexp[p] = phi[ii++];
  int nv = c->lmax + 1 > 2 ? c->lmax + 1 : 2;
#pragma omp parallel
  {
    ref_ws ws;
    ws.basloc = malloc(sizeof(double) * nylm);
    ws.dbsloc = malloc(sizeof(double) * 3 * nylm);
    ws.vplm = malloc(sizeof(double) * nylm);
    ws.vcos = malloc(sizeof(double) * nv);
    ws.vsin = malloc(sizeof(double) * nv);
    /* each sphere writes only its own fx(:,isph): the parallel loop gives the
     * same result as the reference's serial loop (forces_dd.f90:132-136). */
    for (int r = 0; r < nrg; r++) {
      const int i0 = rg[2 * r], i1 = rg[2 * r + 1];
#pragma omp for schedule(dynamic)
      for (int isph = i0; isph < i1; isph++) {
        double *f = fx + 3 * isph;
        f[0] = f[1] = f[2] = 0.0;
        fdoka(c, isph, sigma, xi + (size_t)isph * ngrid, &ws, f);
        fdokb(c, isph, sigma, xi, &ws, f);
        fdoga(c, isph, xi, phiexp, f);
      }
    }
    free(ws.basloc); free(ws.dbsloc); free(ws.vplm); free(ws.vcos); free(ws.vsin);
  }
  double fep = 0.5 * (c->eps - 1.0) / c->eps;
  for (int r = 0; r < nrg; r++)
    for (int k = 3 * rg[2 * r]; k < 3 * rg[2 * r + 1]; k++) fx[k] = fep * fx[k];
  free(xi);
  free(phiexp);
  return 0;
}

/* forces_dd over spheres [i0, i1) only (timing samples). */
int ref_forces_dd_range(const ref_ctx *c, const double *phi, const double *sigma, const double *s,
                        double *fx, int i0, int i1) {
  int rg[2] = {i0, i1};
  return ref_forces_dd_ranges(c, phi, sigma, s, fx, rg, 1);
}

/* ddmkxi / ddmkzeta (ddcosmo.f90:1758-1806). */
void ref_mkxi(const ref_ctx *c, const double *s, double *xi, int zeta) {
  int ii = 0, nylm = c->nylm;
  for (int isph = 0; isph < c->nsph; isph++)
    for (int its = 0; its < c->ngrid; its++) {
      size_t p = (size_t)isph * c->ngrid + its;
      if (c->ui[p] > 0.0) {
        double d = 0.0;
        for (int k = 0; k < nylm; k++) d += c->basis[(size_t)its * nylm + k] * s[(size_t)isph * nylm + k];
        xi[ii++] = c->w[its] * c->ui[p] * d;
      }
    }
  if (zeta) {
    double f = 0.5 * ((c->eps - 1.0) / c->eps);
    for (int k = 0; k < c->ncav; k++) xi[k] = f * xi[k];
  }
}

/* ------------------------------------------------------------------ */
/* solute electrostatics (mkrhs.f90, efld.f90)                          */
/* ------------------------------------------------------------------ */
void ref_mkrhs(int n, const double *charge, const double *x, const double *y, const double *z,
               int ncav, const double *ccav, double *phi, int nylm, double *psi) {
  double pi = 4.0 * atan(1.0), fac = sqrt(4.0 * pi);
#pragma omp parallel for schedule(static)
  for (int ic = 0; ic < ncav; ic++) {
    double v = 0.0;
    for (int j = 0; j < n; j++) {
      double dx = ccav[3 * ic] - x[j], dy = ccav[3 * ic + 1] - y[j], dz = ccav[3 * ic + 2] - z[j];
      double d2 = dx * dx + dy * dy + dz * dz;
      v = v + charge[j] / sqrt(d2);
    }
    phi[ic] = v;
  }
  for (size_t k = 0; k < (size_t)nylm * n; k++) psi[k] = 0.0;
  for (int isph = 0; isph < n; isph++) psi[(size_t)isph * nylm] = fac * charge[isph];
}

void ref_efld(int nsrc, const double *src, const double *csrc, int ntrg, const double *ctrg,
              double *ef) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ntrg; j++) {
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    for (int i = 0; i < nsrc; i++) {
      double dx = ctrg[3 * j] - csrc[3 * i];
      double dy = ctrg[3 * j + 1] - csrc[3 * i + 1];
      double dz = ctrg[3 * j + 2] - csrc[3 * i + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      double rr = sqrt(r2);
      double r3 = r2 * rr;
      double f = src[i] / r3;
      e0 = e0 + f * dx;
      e1 = e1 + f * dy;
      e2 = e2 + f * dz;
    }
    ef[3 * j] = e0;
    ef[3 * j + 1] = e1;
    ef[3 * j + 2] = e2;
  }
}

/* ------------------------------------------------------------------ */
/* the main.f90 energy + forces flow (main.f90:164-265)                 */
/* ------------------------------------------------------------------ */
/* Inputs in bohr.  Outputs: esolv (Hartree), sigma/s (nylm,n), fx(3,n)
 * (total forces, Hartree/bohr), iters[2] (direct, adjoint).
 * Returns 0, or 1/2 when the direct/adjoint solve did not converge. */
int ref_energy_forces(ref_ctx *c, int n, const double *q, const double *x, const double *y,
                      const double *z, const double *r, double *esolv, double *sigma, double *s,
                      double *fx, int *iters) {
  ref_init(c, n, x, y, z, r);
  int ncav = c->ncav, nylm = c->nylm, ngrid = c->ngrid;
  double *phi = malloc(sizeof(double) * (ncav > 0 ? ncav : 1));
  double *psi = malloc(sizeof(double) * (size_t)nylm * n);
  ref_mkrhs(n, q, x, y, z, ncav, c->ccav, phi, nylm, psi);
  int rc = ref_cosmo(c, 0, 1, phi, NULL, psi, sigma, esolv, &iters[0], NULL);
  if (rc) { free(phi); free(psi); return 1; }
  if (c->igrad) {
    double dummy;
    rc = ref_cosmo(c, 1, 0, NULL, NULL, psi, s, &dummy, &iters[1], NULL);
    if (rc) { free(phi); free(psi); return 2; }
    ref_forces_dd(c, phi, sigma, s, fx);
    double *zeta = malloc(sizeof(double) * (ncav > 0 ? ncav : 1));
    ref_mkxi(c, s, zeta, 1);
    int mx = n > ncav ? n : ncav;
    double *ef = malloc(sizeof(double) * 3 * (mx > 0 ? mx : 1));
    ref_efld(n, q, c->csph, ncav, c->ccav, ef);
    int ii = 0;
    for (int isph = 0; isph < n; isph++)
      for (int ig = 0; ig < ngrid; ig++)
        if (c->ui[(size_t)isph * ngrid + ig] > 0.0) {
          for (int k = 0; k < 3; k++) fx[3 * isph + k] = fx[3 * isph + k] - zeta[ii] * ef[3 * ii + k];
          ii++;
        }
    ref_efld(ncav, zeta, c->ccav, n, c->csph, ef);
    for (int isph = 0; isph < n; isph++)
      for (int k = 0; k < 3; k++) fx[3 * isph + k] = fx[3 * isph + k] - ef[3 * isph + k] * q[isph];
    free(zeta);
    free(ef);
  }
  free(phi);
  free(psi);
  return 0;
}

int ref_last_iters(const ref_ctx *c) { return c->last_iters; }

int ref_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
