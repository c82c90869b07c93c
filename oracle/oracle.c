/*
 * CPU oracle: a plain-C restatement of METHOD's per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (method_b200/) links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the
 * CPU-baseline / reference arms of bench.py use it, as the checker.
 *
 * It restates, function by function, the reference's serial CPU code
 * (paths relative to the METHOD repository):
 *   WENO point kernels ....... Project/CPU/Src/wenoUpwinds.cc:5-83
 *   WENO sweeps .............. Project/CPU/Src/weno.cc:23-228
 *   FVS flux method .......... Project/CPU/Src/fluxVectorSplitting.cc:4-131
 *   SRMHD model .............. Project/CPU/Src/srmhd.cc:72-673
 *   SRRMHD model ............. Project/CPU/Src/srrmhd.cc:65-581
 *   Boundary conditions ...... Project/CPU/Src/boundaryConds.cc:5-145, 449-733
 *   RK2 / RKSplit / SSP2 ..... Project/CPU/Src/RK2.cc, rkSplit.cc, SSP2.cc, IMEX2Args.cc
 *   SSP3 / SSP2322 ........... Project/CPU/Src/SSP3.cc, SSP2322.cc, IMEX3Args.cc
 *   Simulation::updateTime ... Project/CPU/Src/simulation.cc:104-133
 *   Powell hybrid (hybrd1) ... Project/CPU/CminpackLibrary/Src/{hybrd1,hybrd,fdjac1,
 *                              qrfac,qform,dogleg,r1updt,r1mpyq,enorm}.cc
 * keeping every floating-point expression in the reference's association
 * order, so that a build without FMA contraction (gcc's x86-64 default)
 * reproduces the reference bit for bit.  That property is what the tests pin
 * (tests/test_oracle_cpu.py) before the oracle is used to check the GPU path.
 *
 * Layout: ID(var,i,j,k) = var*Nx*Ny*Nz + i*Ny*Nz + j*Nz + k (simData.h:10).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int model; /* 0 SRMHD, 1 SRRMHD */
  int nx, ny, nz;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double endTime, cfl;
  int Ng;
  double gamma, sigma, cp;
  int weno;       /* 3, 5, 7, 9 or 11 */
  int bcs;        /* 0 outflow, 1 periodic, 2 flow */
  int integrator; /* 0 RK2, 1 RKSplit, 2 SSP2, 3 SSP3, 4 SSP2322 */
  int functional_sigma; /* Data::functionalSigma */
  double sigma_exp;     /* Data::gam */
} orc_config;

/* Data::sigmaFunc (simData.cc:114-127) of a cell whose density is D. */
static double sigma_func(const orc_config* c, double D) {
  return c->functional_sigma ? c->sigma * pow(D, c->sigma_exp) : c->sigma;
}

typedef struct {
  orc_config c;
  int Nx, Ny, Nz, Ntot, dims, is, ie, js, je, ks, ke;
  int NC, NP, NA;
  double dx, dy, dz, t, dt;
  int iters;
  double *cons, *prims, *aux, *f;
  double *p1cons, *p1prims, *p1aux, *args1, *args2; /* RK2 */
  double *U1, *U2, *flux1, *flux2, *source1, *source2; /* SSP2 */
  double *U3, *flux3, *source3, *tprims, *taux;      /* SSP3 / SSP2322 */
  double *solution;                                   /* SRMHD C2P */
  double *fplus, *fminus, *fprec, *fmrec, *fx, *fy, *fz, *source;
  int failed; /* 1 C2P, 2 implicit */
  int c2p_unconverged; /* SRMHD C2P: cells the last call's retry left unconverged */
} orc_sim;

#define IDX(s, v, i, j, k) ((size_t)(v) * (s)->Ntot + ((size_t)(i) * (s)->Ny + (j)) * (s)->Nz + (k))

/* ------------------------------------------------------------------------ */
/* WENO point kernels (wenoUpwinds.cc:5-83)                                 */

double orc_weno3_upwind(double v0, double v1, double v2) {
  double eps = 1e-16, b0 = 0, b1 = 0, s0 = 0, s1 = 0, a0, a1, sum, w0, w1;
  b0 += 1.0 * v1 * v1;
  b0 += -2.0 * v0 * v1;
  b0 += 1.0 * v0 * v0;
  a0 = 0.3333333333333333 / (eps + b0 * b0);
  b1 += 1.0 * v2 * v2;
  b1 += -2.0 * v1 * v2;
  b1 += 1.0 * v1 * v1;
  a1 = 0.6666666666666666 / (eps + b1 * b1);
  sum = a0 + a1;
  w0 = a0 / sum;
  w1 = a1 / sum;
  s0 += 1.5 * v1;
  s0 += -0.5 * v0;
  s1 += 0.5 * v2;
  s1 += 0.5 * v1;
  return (w0 * s0 + w1 * s1);
}

double orc_weno5_upwind(double v0, double v1, double v2, double v3, double v4) {
  double eps = 1e-16, b0 = 0, b1 = 0, b2 = 0, s0 = 0, s1 = 0, s2 = 0, a0, a1, a2, sum;
  b0 += 3.3333333333333335 * v2 * v2;
  b0 += -10.333333333333334 * v1 * v2;
  b0 += 8.333333333333334 * v1 * v1;
  b0 += 3.6666666666666665 * v0 * v2;
  b0 += -6.333333333333333 * v0 * v1;
  b0 += 1.3333333333333333 * v0 * v0;
  a0 = 0.1 / (eps + b0 * b0);
  b1 += 1.3333333333333333 * v3 * v3;
  b1 += -4.333333333333333 * v2 * v3;
  b1 += 4.333333333333333 * v2 * v2;
  b1 += 1.6666666666666667 * v1 * v3;
  b1 += -4.333333333333333 * v1 * v2;
  b1 += 1.3333333333333333 * v1 * v1;
  a1 = 0.6 / (eps + b1 * b1);
  b2 += 1.3333333333333333 * v4 * v4;
  b2 += -6.333333333333333 * v3 * v4;
  b2 += 8.333333333333334 * v3 * v3;
  b2 += 3.6666666666666665 * v2 * v4;
  b2 += -10.333333333333334 * v2 * v3;
  b2 += 3.3333333333333335 * v2 * v2;
  a2 = 0.3 / (eps + b2 * b2);
  sum = a0 + a1 + a2;
  s0 += 1.8333333333333333 * v2;
  s0 += -1.1666666666666667 * v1;
  s0 += 0.3333333333333333 * v0;
  s1 += 0.3333333333333333 * v3;
  s1 += 0.8333333333333334 * v2;
  s1 += -0.16666666666666666 * v1;
  s2 += -0.16666666666666666 * v4;
  s2 += 0.8333333333333334 * v3;
  s2 += 0.3333333333333333 * v2;
  return (a0 / sum * s0 + a1 / sum * s1 + a2 / sum * s2);
}

/* ------------------------------------------------------------------------ */
/* Powell hybrid method as configured by hybrd1 (hybrd1.cc:114-143).        */
/* Run-time n, 0-based, column-major Jacobian.                              */

typedef void (*orc_fcn)(void* ctx, int n, const double* x, double* f);

static double enorm_n(int n, const double* x) {
  const double rdwarf = 1.82691291192569e-153, rgiant = 1.34078079299426e+153;
  double s1 = 0., s2 = 0., s3 = 0., x1max = 0., x3max = 0., agiant = rgiant / (double)n;
  for (int i = 0; i < n; ++i) {
    double xa = fabs(x[i]), d;
    if (xa >= agiant) {
      if (xa > x1max) { d = x1max / xa; s1 = 1. + s1 * (d * d); x1max = xa; }
      else { d = xa / x1max; s1 += d * d; }
    } else if (xa <= rdwarf) {
      if (xa > x3max) { d = x3max / xa; s3 = 1. + s3 * (d * d); x3max = xa; }
      else if (xa != 0.) { d = xa / x3max; s3 += d * d; }
    } else {
      s2 += xa * xa;
    }
  }
  if (s1 != 0.) return x1max * sqrt(s1 + (s2 / x1max) / x1max);
  if (s2 != 0.) {
    if (s2 >= x3max) return sqrt(s2 * (1. + (x3max / s2) * (x3max * s3)));
    return sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
  }
  return x3max * sqrt(s3);
}

/* packed row-wise upper triangle of an n x n matrix */
static int rp(int n, int i, int j) { return i * n - i * (i - 1) / 2 + (j - i); }

static void dogleg_n(int n, const double* r, const double* qtb, double delta, double* x,
                     double* wa1, double* wa2) {
  double epsmch = DBL_EPSILON, qnorm, gnorm, sgnorm, alpha, temp, sum;
  for (int k = 0; k < n; ++k) {
    int j = n - 1 - k;
    sum = 0.;
    for (int i = j + 1; i < n; ++i) sum += r[rp(n, j, i)] * x[i];
    temp = r[rp(n, j, j)];
    if (temp == 0.) {
      for (int i = 0; i <= j; ++i) { double d2 = fabs(r[rp(n, i, j)]); temp = temp >= d2 ? temp : d2; }
      temp = epsmch * temp;
      if (temp == 0.) temp = epsmch;
    }
    x[j] = (qtb[j] - sum) / temp;
  }
  for (int j = 0; j < n; ++j) { wa1[j] = 0.; wa2[j] = x[j]; }
  qnorm = enorm_n(n, wa2);
  if (qnorm <= delta) return;
  for (int j = 0; j < n; ++j) {
    temp = qtb[j];
    for (int i = j; i < n; ++i) wa1[i] += r[rp(n, j, i)] * temp;
  }
  gnorm = enorm_n(n, wa1);
  sgnorm = 0.;
  alpha = delta / qnorm;
  if (gnorm != 0.) {
    for (int j = 0; j < n; ++j) wa1[j] = wa1[j] / gnorm;
    for (int j = 0; j < n; ++j) {
      sum = 0.;
      for (int i = j; i < n; ++i) sum += r[rp(n, j, i)] * wa1[i];
      wa2[j] = sum;
    }
    temp = enorm_n(n, wa2);
    sgnorm = gnorm / temp / temp;
    alpha = 0.;
    if (sgnorm < delta) {
      double bnorm = enorm_n(n, qtb), d1, d2, d3, d4;
      temp = bnorm / gnorm * (bnorm / qnorm) * (sgnorm / delta);
      d1 = sgnorm / delta;
      d2 = temp - delta / qnorm;
      d3 = delta / qnorm;
      d4 = sgnorm / delta;
      temp = temp - delta / qnorm * (d1 * d1) + sqrt(d2 * d2 + (1. - d3 * d3) * (1. - d4 * d4));
      d1 = sgnorm / delta;
      alpha = delta / qnorm * (1. - d1 * d1) / temp;
    }
  }
  temp = (1. - alpha) * (sgnorm <= delta ? sgnorm : delta);
  for (int j = 0; j < n; ++j) x[j] = temp * wa1[j] + alpha * x[j];
}

static void rot_from(double num, double den, int swap, double* c, double* s, double* tau) {
  if (swap) {
    double ct = den / num;
    *s = .5 / sqrt(.25 + .25 * (ct * ct));
    *c = *s * ct;
    *tau = 1.;
    if (fabs(*c) * DBL_MAX > 1.) *tau = 1. / *c;
  } else {
    double tn = num / den;
    *c = .5 / sqrt(.25 + .25 * (tn * tn));
    *s = *c * tn;
    *tau = *s;
  }
}

static void r1updt_n(int n, double* s, const double* u, double* v, double* w) {
  w[n - 1] = s[rp(n, n - 1, n - 1)];
  for (int j = n - 2; j >= 0; --j) {
    w[j] = 0.;
    if (v[j] != 0.) {
      double c, sn, tau;
      rot_from(v[j], v[n - 1], fabs(v[n - 1]) < fabs(v[j]), &c, &sn, &tau);
      v[n - 1] = sn * v[j] + c * v[n - 1];
      v[j] = tau;
      for (int i = j; i < n; ++i) {
        double t = c * s[rp(n, j, i)] - sn * w[i];
        w[i] = sn * s[rp(n, j, i)] + c * w[i];
        s[rp(n, j, i)] = t;
      }
    }
  }
  for (int i = 0; i < n; ++i) w[i] += v[n - 1] * u[i];
  for (int j = 0; j < n - 1; ++j) {
    if (w[j] != 0.) {
      double c, sn, tau;
      rot_from(w[j], s[rp(n, j, j)], fabs(s[rp(n, j, j)]) < fabs(w[j]), &c, &sn, &tau);
      for (int i = j; i < n; ++i) {
        double t = c * s[rp(n, j, i)] + sn * w[i];
        w[i] = -sn * s[rp(n, j, i)] + c * w[i];
        s[rp(n, j, i)] = t;
      }
      w[j] = tau;
    }
  }
  s[rp(n, n - 1, n - 1)] = w[n - 1];
}

static void unrot(double t, double* c, double* s) {
  if (fabs(t) > 1.) { *c = 1. / t; *s = sqrt(1. - *c * *c); }
  else { *s = t; *c = sqrt(1. - *s * *s); }
}

/* a is m x n column-major with leading dimension lda */
static void r1mpyq_n(int m, int n, double* a, int lda, const double* v, const double* w) {
  for (int j = n - 2; j >= 0; --j) {
    double c, s;
    unrot(v[j], &c, &s);
    for (int i = 0; i < m; ++i) {
      double t = c * a[i + lda * j] - s * a[i + lda * (n - 1)];
      a[i + lda * (n - 1)] = s * a[i + lda * j] + c * a[i + lda * (n - 1)];
      a[i + lda * j] = t;
    }
  }
  for (int j = 0; j < n - 1; ++j) {
    double c, s;
    unrot(w[j], &c, &s);
    for (int i = 0; i < m; ++i) {
      double t = c * a[i + lda * j] + s * a[i + lda * (n - 1)];
      a[i + lda * (n - 1)] = -s * a[i + lda * j] + c * a[i + lda * (n - 1)];
      a[i + lda * j] = t;
    }
  }
}

/* Returns MINPACK's info (1 converged; 2, 3, 4 failures; 5 mapped to 4). */
int orc_hybrd1(orc_fcn fcn, void* ctx, int n, double* x, double* fvec, double tol, int* nfev_out) {
  if (n <= 0 || tol < 0.) return 0;
  const int maxfev = 200 * (n + 1);
  const double epsmch = tol * tol, factor = 100.;
  double* fjac = (double*)malloc(sizeof(double) * (n * n + n * (n + 1) / 2 + 6 * n));
  double* r = fjac + n * n;
  double* qtf = r + n * (n + 1) / 2;
  double *wa1 = qtf + n, *wa2 = wa1 + n, *wa3 = wa2 + n, *wa4 = wa3 + n;
  int nfev, iter = 1, ncsuc = 0, ncfail = 0, nslow1 = 0, nslow2 = 0, info = 0;
  double fnorm, delta = 0., xnorm = 0.;

  fcn(ctx, n, x, fvec);
  nfev = 1;
  fnorm = enorm_n(n, fvec);
  for (;;) {
    int jeval = 1;
    for (int j = 0; j < n; ++j) { /* fdjac1, dense */
      double temp = x[j], h = 1.414213562373095e-08 * fabs(temp);
      if (h < 1.0e-17) h = 1.414213562373095e-08;
      x[j] = temp + h;
      fcn(ctx, n, x, wa1);
      x[j] = temp;
      for (int i = 0; i < n; ++i) fjac[i + n * j] = (wa1[i] - fvec[i]) / h;
    }
    nfev += n;
    for (int j = 0; j < n; ++j) { /* qrfac, no pivoting */
      double ajnorm = enorm_n(n - j, fjac + j + n * j);
      if (ajnorm != 0.) {
        if (fjac[j + n * j] < 0.) ajnorm = -ajnorm;
        for (int i = j; i < n; ++i) fjac[i + n * j] /= ajnorm;
        fjac[j + n * j] += 1.;
        for (int k = j + 1; k < n; ++k) {
          double sum = 0., temp;
          for (int i = j; i < n; ++i) sum += fjac[i + n * j] * fjac[i + n * k];
          temp = sum / fjac[j + n * j];
          for (int i = j; i < n; ++i) fjac[i + n * k] -= temp * fjac[i + n * j];
        }
      }
      wa1[j] = -ajnorm;
    }
    if (iter == 1) {
      for (int j = 0; j < n; ++j) wa3[j] = x[j];
      xnorm = enorm_n(n, wa3);
      delta = factor * xnorm;
      if (delta == 0.) delta = factor;
    }
    for (int i = 0; i < n; ++i) qtf[i] = fvec[i];
    for (int j = 0; j < n; ++j) {
      if (fjac[j + n * j] != 0.) {
        double sum = 0., temp;
        for (int i = j; i < n; ++i) sum += fjac[i + n * j] * qtf[i];
        temp = -sum / fjac[j + n * j];
        for (int i = j; i < n; ++i) qtf[i] += fjac[i + n * j] * temp;
      }
    }
    for (int j = 0; j < n; ++j) {
      for (int i = 0; i < j; ++i) r[rp(n, i, j)] = fjac[i + n * j];
      r[rp(n, j, j)] = wa1[j];
    }
    for (int j = 1; j < n; ++j) /* qform */
      for (int i = 0; i < j; ++i) fjac[i + n * j] = 0.;
    for (int k = n - 1; k >= 0; --k) {
      for (int i = k; i < n; ++i) { wa1[i] = fjac[i + n * k]; fjac[i + n * k] = 0.; }
      fjac[k + n * k] = 1.;
      if (wa1[k] != 0.) {
        for (int j = k; j < n; ++j) {
          double sum = 0., temp;
          for (int i = k; i < n; ++i) sum += fjac[i + n * j] * wa1[i];
          temp = sum / wa1[k];
          for (int i = k; i < n; ++i) fjac[i + n * j] -= temp * wa1[i];
        }
      }
    }
    for (;;) {
      double pnorm, fnorm1, actred, prered, ratio, temp;
      dogleg_n(n, r, qtf, delta, wa1, wa2, wa3);
      for (int j = 0; j < n; ++j) { wa1[j] = -wa1[j]; wa2[j] = x[j] + wa1[j]; wa3[j] = wa1[j]; }
      pnorm = enorm_n(n, wa3);
      if (iter == 1) delta = delta <= pnorm ? delta : pnorm;
      fcn(ctx, n, wa2, wa4);
      ++nfev;
      fnorm1 = enorm_n(n, wa4);
      actred = -1.;
      if (fnorm1 < fnorm) { double d1 = fnorm1 / fnorm; actred = 1. - d1 * d1; }
      for (int i = 0; i < n; ++i) {
        double sum = 0.;
        for (int j = i; j < n; ++j) sum += r[rp(n, i, j)] * wa1[j];
        wa3[i] = qtf[i] + sum;
      }
      temp = enorm_n(n, wa3);
      prered = 0.;
      if (temp < fnorm) { double d1 = temp / fnorm; prered = 1. - d1 * d1; }
      ratio = 0.;
      if (prered > 0.) ratio = actred / prered;
      if (ratio < .1) {
        ncsuc = 0;
        ++ncfail;
        delta = .5 * delta;
      } else {
        ncfail = 0;
        ++ncsuc;
        if (ratio >= .5 || ncsuc > 1) { double d1 = pnorm / .5; delta = delta >= d1 ? delta : d1; }
        if (fabs(ratio - 1.) <= .1) delta = pnorm / .5;
      }
      if (ratio >= 1e-4) {
        for (int j = 0; j < n; ++j) { x[j] = wa2[j]; wa2[j] = x[j]; fvec[j] = wa4[j]; }
        xnorm = enorm_n(n, wa2);
        fnorm = fnorm1;
        ++iter;
      }
      ++nslow1;
      if (actred >= .001) nslow1 = 0;
      if (jeval) ++nslow2;
      if (actred >= .1) nslow2 = 0;
      if (delta <= tol * xnorm || fnorm == 0.) info = 1;
      if (info) goto done;
      if (nfev >= maxfev) info = 2;
      { double d1 = .1 * delta; if (.1 * (d1 >= pnorm ? d1 : pnorm) <= epsmch * xnorm) info = 3; }
      if (nslow2 == 5) info = 4;
      if (nslow1 == 10) info = 5;
      if (info) goto done;
      if (ncfail == 2) break;
      for (int j = 0; j < n; ++j) {
        double sum = 0.;
        for (int i = 0; i < n; ++i) sum += fjac[i + n * j] * wa4[i];
        wa2[j] = (sum - wa3[j]) / pnorm;
        wa1[j] = wa1[j] / pnorm;
        if (ratio >= 1e-4) qtf[j] = sum;
      }
      r1updt_n(n, r, wa1, wa2, wa3);
      r1mpyq_n(n, n, fjac, n, wa2, wa3);
      r1mpyq_n(1, n, qtf, 1, wa2, wa3);
      jeval = 0;
    }
  }
done:
  free(fjac);
  if (nfev_out) *nfev_out = nfev;
  return info == 5 ? 4 : info;
}

/* Known-answer systems of Tests/CPU/Src/test_cminpack.cc:5-29. */
static void kat_fcn(void* ctx, int n, const double* x, double* f) {
  int which = *(int*)ctx;
  (void)n;
  if (which == 0) { f[0] = (x[0] + 4) * (x[0] + 4) * (x[0] + 4); f[1] = (x[1] - 2.5) * (x[1] - 2.5); }
  else if (which == 1) { f[0] = x[0] * x[0] + 5.0; f[1] = -x[1] * x[1] - 5.0; }
  else { f[0] = exp(x[0]) + x[0] * x[1] - 1; f[1] = sin(x[0] * x[1]) + x[0] + x[1] - 1; }
}

int orc_hybrd1_kat(int which, int n, double* x, double* fvec, double tol, int lwa) {
  if (lwa < n * (n * 3 + 13) / 2) return 0;
  return orc_hybrd1(kat_fcn, &which, n, x, fvec, tol, NULL);
}

/* ------------------------------------------------------------------------ */
/* SRMHD (srmhd.cc)                                                          */

static void srmhd_flux_cell(const double* c, const double* p, const double* a, int dir, double* f) {
  if (dir == 0) {
    f[0] = c[0] * p[1];
    f[1] = c[1] * p[1] + (p[4] + a[8] * 0.5) - a[5] * p[5] / a[1];
    f[2] = c[2] * p[1] - a[6] * p[5] / a[1];
    f[3] = c[3] * p[1] - a[7] * p[5] / a[1];
    f[4] = (c[4] + p[4] + a[8] * 0.5) * p[1] - a[4] * p[5] / a[1];
    f[5] = c[8];
    f[6] = p[6] * p[1] - p[5] * p[2];
    f[7] = p[7] * p[1] - p[5] * p[3];
    f[8] = p[5];
  } else if (dir == 1) {
    f[0] = c[0] * p[2];
    f[1] = c[1] * p[2] - a[5] * p[6] / a[1];
    f[2] = c[2] * p[2] + p[4] + a[8] * 0.5 - a[6] * p[6] / a[1];
    f[3] = c[3] * p[2] - a[7] * p[6] / a[1];
    f[4] = (c[4] + p[4] + a[8] * 0.5) * p[2] - a[4] * p[6] / a[1];
    f[5] = p[5] * p[2] - p[6] * p[1];
    f[6] = c[8];
    f[7] = p[7] * p[2] - p[6] * p[3];
    f[8] = p[6];
  } else {
    f[0] = c[0] * p[3];
    f[1] = c[1] * p[3] - a[5] * p[7] / a[1];
    f[2] = c[2] * p[3] - a[6] * p[7] / a[1];
    f[3] = c[3] * p[3] + p[4] + a[8] * 0.5 - a[7] * p[7] / a[1];
    f[4] = (c[4] + p[4] + a[8] * 0.5) * p[3] - a[4] * p[7] / a[1];
    f[5] = p[5] * p[3] - p[7] * p[1];
    f[6] = p[6] * p[3] - p[7] * p[2];
    f[7] = c[8];
    f[8] = p[6];
  }
}

typedef struct { double D, g, BS, Bsq, Ssq, tau; } srmhd_args;

static void srmhd_residual(void* ctx, int n, const double* x, double* f) {
  srmhd_args* a = (srmhd_args*)ctx;
  double W, rho, h, pr;
  (void)n;
  if (x[0] >= 1.0 || x[1] < 0) { f[0] = f[1] = 1e6; return; }
  W = 1 / sqrt(1 - x[0]);
  rho = a->D / W;
  h = x[1] / (rho * W * W);
  pr = (h - 1) * rho * (a->g - 1) / a->g;
  if (pr < 0 || rho < 0 || h < 0 || W < 1) { f[0] = f[1] = 1e6; return; }
  f[0] = (x[1] + a->Bsq) * (x[1] + a->Bsq) * x[0] - (2 * x[1] + a->Bsq) * a->BS * a->BS / (x[1] * x[1]) - a->Ssq;
  f[1] = x[1] + a->Bsq - pr - a->Bsq / (2 * W * W) - a->BS * a->BS / (2 * x[1] * x[1]) - a->D - a->tau;
}

static void srmhd_closed_form(orc_sim* s, const double* cons, double* prims, double* aux, int i, int j, int k) {
  double g = s->c.gamma, *sol = s->solution;
#define C(v) cons[IDX(s, v, i, j, k)]
#define P(v) prims[IDX(s, v, i, j, k)]
#define A(v) aux[IDX(s, v, i, j, k)]
#define SOL(v) sol[IDX(s, v, i, j, k)]
  A(1) = 1 / sqrt(1 - SOL(0));
  P(0) = C(0) / A(1);
  A(0) = SOL(1) / (P(0) * A(1) * A(1));
  P(4) = (A(0) - 1) * P(0) * (g - 1) / g;
  A(2) = P(4) / (P(0) * (g - 1));
  P(1) = (C(5) * A(10) + C(1) * SOL(1)) / (SOL(1) * (A(11) + SOL(1)));
  P(2) = (C(6) * A(10) + C(2) * SOL(1)) / (SOL(1) * (A(11) + SOL(1)));
  P(3) = (C(7) * A(10) + C(3) * SOL(1)) / (SOL(1) * (A(11) + SOL(1)));
  A(9) = P(1) * P(1) + P(2) * P(2) + P(3) * P(3);
  A(3) = sqrt(A(2) * g * (g - 1) / A(0));
  A(4) = A(1) * (C(5) * P(1) + C(6) * P(2) + C(7) * P(3));
  A(5) = C(5) / A(1) + A(4) * P(1);
  A(6) = C(6) / A(1) + A(4) * P(2);
  A(7) = C(7) / A(1) + A(4) * P(3);
  A(8) = (P(5) * P(5) + P(6) * P(6) + P(7) * P(7) + A(4) * A(4)) / (A(1) * A(1));
}

/* SRMHD::getPrimitiveVars (srmhd.cc:390-562), including the neighbour-average
 * retry that reuses the residual arguments of the last interior cell. */
static void srmhd_c2p(orc_sim* s, double* cons, double* prims, double* aux) {
  const double tol = 1.49011612e-7;
  srmhd_args args;
  double sol[2], res[2];
  int* fails = NULL;
  int nf = 0, cap = 0;
  memset(&args, 0, sizeof args);
  s->c2p_unconverged = 0;
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) {
        P(5) = C(5); P(6) = C(6); P(7) = C(7);
        A(10) = C(5) * C(1) + C(6) * C(2) + C(7) * C(3);
        A(11) = C(5) * C(5) + C(6) * C(6) + C(7) * C(7);
        A(12) = C(1) * C(1) + C(2) * C(2) + C(3) * C(3);
        args.D = C(0); args.g = s->c.gamma; args.BS = A(10); args.Bsq = A(11); args.Ssq = A(12);
        args.tau = C(4);
        sol[0] = P(1) * P(1) + P(2) * P(2) + P(3) * P(3);
        sol[1] = P(0) * A(0) / (1 - sol[0]);
        if (orc_hybrd1(srmhd_residual, &args, 2, sol, res, tol, NULL) != 1) {
          if (nf == cap) { cap = cap ? 2 * cap : 64; fails = (int*)realloc(fails, sizeof(int) * 3 * cap); }
          fails[3 * nf] = i; fails[3 * nf + 1] = j; fails[3 * nf + 2] = k; nf++;
        } else {
          s->solution[IDX(s, 0, i, j, k)] = sol[0];
          s->solution[IDX(s, 1, i, j, k)] = sol[1];
        }
      }
  for (int f = 0; f < nf; ++f) {
    int x = fails[3 * f], y = fails[3 * f + 1], z = fails[3 * f + 2], cnt = 0;
    int nb[6][3];
    if (x > 0) { nb[cnt][0] = x - 1; nb[cnt][1] = y; nb[cnt++][2] = z; }
    if (y > 0) { nb[cnt][0] = x; nb[cnt][1] = y - 1; nb[cnt++][2] = z; }
    if (z > 0) { nb[cnt][0] = x; nb[cnt][1] = y; nb[cnt++][2] = z - 1; }
    if (x < s->Nx - 1) { nb[cnt][0] = x + 1; nb[cnt][1] = y; nb[cnt++][2] = z; }
    if (y < s->Ny - 1) { nb[cnt][0] = x; nb[cnt][1] = y + 1; nb[cnt++][2] = z; }
    if (z < s->Nz - 1) { nb[cnt][0] = x; nb[cnt][1] = y; nb[cnt++][2] = z + 1; }
    sol[0] = 0; sol[1] = 0;
    for (int q = 0; q < cnt; ++q) {
      sol[0] += s->solution[IDX(s, 0, nb[q][0], nb[q][1], nb[q][2])];
      sol[1] += s->solution[IDX(s, 1, nb[q][0], nb[q][1], nb[q][2])];
    }
    sol[0] /= (double)cnt;
    sol[1] /= (double)cnt;
    if (orc_hybrd1(srmhd_residual, &args, 2, sol, res, tol, NULL) != 1) s->c2p_unconverged++;
    s->solution[IDX(s, 0, x, y, z)] = sol[0];
    s->solution[IDX(s, 1, x, y, z)] = sol[1];
  }
  free(fails);
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) srmhd_closed_form(s, cons, prims, aux, i, j, k);
}

static void srmhd_prims_to_all(orc_sim* s, double* cons, double* prims, double* aux) {
  double g = s->c.gamma;
  for (int i = 0; i < s->Nx; i++)
    for (int j = 0; j < s->Ny; j++)
      for (int k = 0; k < s->Nz; k++) {
        C(5) = P(5); C(6) = P(6); C(7) = P(7);
        A(11) = P(5) * P(5) + P(6) * P(6) + P(7) * P(7);
        C(8) = 0;
        A(9) = P(1) * P(1) + P(2) * P(2) + P(3) * P(3);
        A(1) = 1.0 / sqrt(1 - A(9));
        A(4) = A(1) * (P(1) * P(5) + P(2) * P(6) + P(3) * P(7));
        A(5) = P(5) / A(1) + A(4) * P(1);
        A(6) = P(6) / A(1) + A(4) * P(2);
        A(7) = P(7) / A(1) + A(4) * P(3);
        A(8) = (P(5) * P(5) + P(6) * P(6) + P(7) * P(7) + A(4) * A(4)) / (A(1) * A(1));
        A(0) = 1 + P(4) / P(0) * (g / (g - 1));
        A(2) = P(4) / (P(0) * (g - 1));
        A(3) = sqrt(A(2) * g * (g - 1) / A(0));
        C(0) = P(0) * A(1);
        C(1) = (P(0) * A(0) + A(8)) * A(1) * A(1) * P(1) - A(4) * A(5);
        C(2) = (P(0) * A(0) + A(8)) * A(1) * A(1) * P(2) - A(4) * A(6);
        C(3) = (P(0) * A(0) + A(8)) * A(1) * A(1) * P(3) - A(4) * A(7);
        A(12) = C(1) * C(1) + C(2) * C(2) + C(3) * C(3);
        A(10) = P(5) * C(1) + P(6) * C(2) + P(7) * C(3);
        C(4) = (P(0) * A(0) + A(8)) * A(1) * A(1) - (P(4) + A(8) / 2.0) - A(4) * A(4) - C(0);
      }
}

/* ------------------------------------------------------------------------ */
/* SRRMHD (srrmhd.cc)                                                        */

static void srrmhd_flux_cell(const double* c, const double* p, const double* a, int dir, double* f) {
  if (dir == 0) {
    f[0] = c[0] * p[1];
    f[1] = a[10] * p[1] * p[1] + p[4] - c[8] * c[8] - c[5] * c[5] + 0.5 * (a[7] + a[8]);
    f[2] = a[10] * p[1] * p[2] - c[8] * c[9] - c[5] * c[6];
    f[3] = a[10] * p[1] * p[3] - c[8] * c[10] - c[5] * c[7];
    f[4] = c[1] - c[0] * p[1];
    f[5] = c[12]; f[6] = -c[10]; f[7] = c[9];
    f[8] = c[11]; f[9] = c[7]; f[10] = -c[6];
    f[11] = c[8]; f[12] = c[5]; f[13] = a[4];
  } else if (dir == 1) {
    f[0] = c[0] * p[2];
    f[1] = a[10] * p[1] * p[2] - c[9] * c[8] - c[6] * c[5];
    f[2] = a[10] * p[2] * p[2] + p[4] - c[9] * c[9] - c[6] * c[6] + 0.5 * (a[7] + a[8]);
    f[3] = a[10] * p[2] * p[3] - c[9] * c[10] - c[6] * c[7];
    f[4] = c[2] - c[0] * p[2];
    f[5] = c[10]; f[6] = c[12]; f[7] = -c[8];
    f[8] = -c[7]; f[9] = c[11]; f[10] = c[5];
    f[11] = c[9]; f[12] = c[6]; f[13] = a[5];
  } else {
    /* the reference's z branch overwrites f[2] and keeps f[3] from the y call */
    f[0] = c[0] * p[3];
    f[1] = a[10] * p[1] * p[3] - c[10] * c[8] - c[7] * c[5];
    f[2] = a[10] * p[3] * p[3] + p[4] - c[10] * c[10] - c[7] * c[7] + 0.5 * (a[7] + a[8]);
    f[3] = a[10] * p[2] * p[3] - c[9] * c[10] - c[6] * c[7];
    f[4] = c[3] - c[0] * p[3];
    f[5] = -c[9]; f[6] = c[8]; f[7] = c[12];
    f[8] = c[6]; f[9] = -c[5]; f[10] = c[11];
    f[11] = c[10]; f[12] = c[7]; f[13] = a[6];
  }
}

static void srrmhd_source_cell(const double* c, const double* a, double cp, double* s) {
  s[0] = s[1] = s[2] = s[3] = s[4] = s[5] = s[6] = s[7] = s[13] = 0.0;
  s[8] = -a[4];
  s[9] = -a[5];
  s[10] = -a[6];
  s[11] = c[13] - c[11] / (cp * cp);
  s[12] = -c[12] / (cp * cp);
}

static double srrmhd_zres(double Z, double Ssq, double D, double tauT, double g) {
  double vsq = Ssq / (Z * Z), W, rho, h, p;
  if (vsq >= 1.0 || Z < 0) return 1.0e6;
  W = 1 / sqrt(1 - vsq);
  rho = D / W;
  h = Z / (rho * W * W);
  p = (g - 1) * (h - rho) / g;
  if (rho < 0 || p < 0 || W < 1 || h < 0) return 1.0e6;
  return (1 - (g - 1) / (W * W * g)) * Z + ((g - 1) / (W * g) - 1) * D - tauT;
}

/* secant iteration named `newton` in the reference (srrmhd.cc:539-581) */
static int srrmhd_secant(double* Z, double Ssq, double D, double tauT, double g) {
  double x0 = *Z, x1 = x0 + 1.0e-4, x2, f0, f1, bestX, bestF;
  f0 = srrmhd_zres(x0, Ssq, D, tauT, g);
  f1 = srrmhd_zres(x1, Ssq, D, tauT, g);
  bestX = x0; bestF = f0;
  for (int it = 0; it < 50; it++) {
    if (fabs(f0) < 1.0e-12) { *Z = x0; return 1; }
    x2 = x1 - f1 * (x1 - x0) / (f1 - f0);
    x1 = x0; x0 = x2; f1 = f0;
    f0 = srrmhd_zres(x0, Ssq, D, tauT, g);
    if (fabs(f0) < fabs(bestF)) { bestX = x0; bestF = f0; }
  }
  *Z = bestX;
  return 0;
}

/* getPrimitiveVarsSingleCell (srrmhd.cc:256-312); a[10] holds the guess in
 * and the solution out.  Returns 0 when the secant iteration failed. */
static int srrmhd_c2p_cell(const double* c, double g, double sigma, double* p, double* a) {
  p[5] = c[5]; p[6] = c[6]; p[7] = c[7]; p[8] = c[8]; p[9] = c[9]; p[10] = c[10];
  a[7] = c[5] * c[5] + c[6] * c[6] + c[7] * c[7];
  a[8] = c[8] * c[8] + c[9] * c[9] + c[10] * c[10];
  a[12] = c[1] - (c[9] * c[7] - c[10] * c[6]);
  a[13] = c[2] - (c[10] * c[5] - c[8] * c[7]);
  a[14] = c[3] - (c[8] * c[6] - c[9] * c[5]);
  a[15] = a[12] * a[12] + a[13] * a[13] + a[14] * a[14];
  a[16] = c[4] - 0.5 * (a[7] + a[8]);
  if (!srrmhd_secant(&a[10], a[15], c[0], a[16], g)) return 0;
  a[9] = a[15] / (a[10] * a[10]);
  a[1] = 1.0 / sqrt(1 - a[9]);
  p[0] = c[0] / a[1];
  a[0] = a[10] / (p[0] * a[1] * a[1]);
  a[2] = (a[0] - 1) / g;
  a[3] = sqrt((a[2] * g * (g - 1)) / a[0]);
  p[4] = p[0] * a[2] * (g - 1);
  p[1] = a[12] / a[10];
  p[2] = a[13] / a[10];
  p[3] = a[14] / a[10];
  a[11] = p[1] * c[8] + p[2] * c[9] + p[3] * c[10];
  a[4] = c[13] * p[1] + a[1] * sigma * (c[8] + (p[2] * c[7] - p[3] * c[6]) - a[11] * p[1]);
  a[5] = c[13] * p[2] + a[1] * sigma * (c[9] + (p[3] * c[5] - p[1] * c[7]) - a[11] * p[2]);
  a[6] = c[13] * p[3] + a[1] * sigma * (c[10] + (p[1] * c[6] - p[2] * c[5]) - a[11] * p[3]);
  return 1;
}

static int srrmhd_c2p(orc_sim* s, double* cons, double* prims, double* aux) {
  double c[14], p[11], a[17];
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) {
        for (int v = 0; v < 14; v++) c[v] = C(v);
        a[10] = A(10);
        if (!srrmhd_c2p_cell(c, s->c.gamma, sigma_func(&s->c, c[0]), p, a)) return 1;
        for (int v = 0; v < 11; v++) P(v) = p[v];
        for (int v = 0; v < 17; v++) A(v) = a[v];
      }
  return 0;
}

static void srrmhd_prims_to_all(orc_sim* s, double* cons, double* prims, double* aux) {
  double g = s->c.gamma, sg, dx = s->dx, dy = s->dy, dz = s->dz;
#define PN(v, a, b, cc) prims[IDX(s, v, a, b, cc)]
  for (int i = 0; i < s->Nx; i++)
    for (int j = 0; j < s->Ny; j++)
      for (int k = 0; k < s->Nz; k++) {
        int fd = 1;
        C(11) = C(12) = 0.0;
        C(5) = P(5); C(6) = P(6); C(7) = P(7);
        C(8) = P(8); C(9) = P(9); C(10) = P(10);
        A(7) = P(5) * P(5) + P(6) * P(6) + P(7) * P(7);
        A(8) = P(8) * P(8) + P(9) * P(9) + P(10) * P(10);
        A(9) = P(1) * P(1) + P(2) * P(2) + P(3) * P(3);
        A(11) = P(1) * C(8) + P(2) * C(9) + P(3) * C(10);
        A(1) = 1.0 / sqrt(1 - A(9));
        C(0) = P(0) * A(1);
        A(2) = P(4) / (P(0) * (g - 1));
        A(0) = 1 + A(2) * g;
        A(3) = sqrt((A(2) * g * (g - 1)) / A(0));
        A(10) = P(0) * A(0) * A(1) * A(1);
        sg = sigma_func(&s->c, C(0)); /* srrmhd.cc:410, after D is set */
        if (i > 1 && j > 1 && k > 1 && i < s->Nx - 2 && j < s->Ny - 2 && k < s->Nz - 2) {
          C(13) = (-PN(8, i + 2, j, k) + 8 * PN(8, i + 1, j, k) - 8 * PN(8, i - 1, j, k) + PN(8, i - 2, j, k)) / (12 * dx) +
                  (-PN(9, i, j + 2, k) + 8 * PN(9, i, j + 1, k) - 8 * PN(9, i, j - 1, k) + PN(9, i, j - 2, k)) / (12 * dy) +
                  (-PN(10, i, j, k + 2) + 8 * PN(10, i, j, k + 1) - 8 * PN(10, i, j, k - 1) + PN(10, i, j, k - 2)) / (12 * dz);
        } else if (i > 1 && j > 1 && i < s->Nx - 2 && j < s->Ny - 2 && s->c.nz == 0) {
          C(13) = (-PN(8, i + 2, j, k) + 8 * PN(8, i + 1, j, k) - 8 * PN(8, i - 1, j, k) + PN(8, i - 2, j, k)) / (12 * dx) +
                  (-PN(9, i, j + 2, k) + 8 * PN(9, i, j + 1, k) - 8 * PN(9, i, j - 1, k) + PN(9, i, j - 2, k)) / (12 * dy);
        } else if (i > 1 && i < s->Nx - 2 && s->c.ny == 0) {
          C(13) = (-PN(8, i + 2, j, k) + 8 * PN(8, i + 1, j, k) - 8 * PN(8, i - 1, j, k) + PN(8, i - 2, j, k)) / (12 * dx);
        } else {
          fd = 0;
          C(13) = A(4) = A(5) = A(6) = 0.0;
        }
        if (fd) {
          A(4) = C(13) * P(1) + A(1) * sg * (C(8) + P(2) * C(7) - P(3) * C(6) - A(11) * P(1));
          A(5) = C(13) * P(2) + A(1) * sg * (C(9) + P(3) * C(5) - P(1) * C(7) - A(11) * P(2));
          A(6) = C(13) * P(3) + A(1) * sg * (C(10) + P(1) * C(6) - P(2) * C(5) - A(11) * P(3));
        }
        C(1) = A(10) * P(1) + C(9) * C(7) - C(10) * C(6);
        C(2) = A(10) * P(2) + C(10) * C(5) - C(8) * C(7);
        C(3) = A(10) * P(3) + C(8) * C(6) - C(9) * C(5);
        C(4) = A(10) - P(4) + 0.5 * (A(7) + A(8)) - C(0);
        A(12) = A(10) * P(1);
        A(13) = A(10) * P(2);
        A(14) = A(10) * P(3);
        A(15) = A(12) * A(12) + A(13) * A(13) + A(14) * A(14);
        A(16) = A(10) - P(4) - C(0);
      }
#undef PN
}

/* ------------------------------------------------------------------------ */
/* Boundary conditions (boundaryConds.cc): x pass, then y, then z.           */

static void bc_arr(orc_sim* s, double* u, int nv) {
  int per_x = s->c.bcs != 0, per_yz = s->c.bcs == 1, Ng = s->c.Ng;
  int nx = s->c.nx, ny = s->c.ny, nz = s->c.nz;
  if (!u) return;
  for (int v = 0; v < nv; v++)
    for (int i = 0; i < Ng; i++)
      for (int j = 0; j < s->Ny; j++)
        for (int k = 0; k < s->Nz; k++) {
          u[IDX(s, v, i, j, k)] = u[IDX(s, v, per_x ? nx + i : Ng, j, k)];
          u[IDX(s, v, nx + Ng + i, j, k)] = u[IDX(s, v, per_x ? Ng + i : nx + Ng - 1, j, k)];
        }
  if (s->Ny > 1)
    for (int v = 0; v < nv; v++)
      for (int i = 0; i < s->Nx; i++)
        for (int j = 0; j < Ng; j++)
          for (int k = 0; k < s->Nz; k++) {
            u[IDX(s, v, i, j, k)] = u[IDX(s, v, i, per_yz ? ny + j : Ng, k)];
            u[IDX(s, v, i, ny + Ng + j, k)] = u[IDX(s, v, i, per_yz ? Ng + j : ny + Ng - 1, k)];
          }
  if (s->Nz > 1)
    for (int v = 0; v < nv; v++)
      for (int i = 0; i < s->Nx; i++)
        for (int j = 0; j < s->Ny; j++)
          for (int k = 0; k < Ng; k++) {
            u[IDX(s, v, i, j, k)] = u[IDX(s, v, i, j, per_yz ? nz + k : Ng)];
            u[IDX(s, v, i, j, nz + Ng + k)] = u[IDX(s, v, i, j, per_yz ? Ng + k : nz + Ng - 1)];
          }
}

void orc_apply_bcs(void* h, double* cons, double* prims, double* aux) {
  orc_sim* s = (orc_sim*)h;
  bc_arr(s, cons, s->NC);
  bc_arr(s, prims, s->NP);
  bc_arr(s, aux, s->NA);
}

/* WENO7 / WENO9 / WENO11 point kernels (wenoUpwinds.cc:86-482), generated
 * by method_b200/gen_weno.py from the Jiang-Shu scheme in exact arithmetic. */
#include "weno_hi.h"

/* The upwind point kernel of order 3 .. 11 on v[0 .. order-1]. */
static double weno_point(int order, const double* v) {
  switch (order) {
    case 3: return orc_weno3_upwind(v[0], v[1], v[2]);
    case 5: return orc_weno5_upwind(v[0], v[1], v[2], v[3], v[4]);
    case 7: return orc_weno7(v[0], v[1], v[2], v[3], v[4], v[5], v[6]);
    case 9: return orc_weno9(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8]);
    default: return orc_weno11(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10]);
  }
}

/* ------------------------------------------------------------------------ */
/* FVS::F (fluxVectorSplitting.cc:4-131) with WENO sweeps (weno.cc).         */

static void flux_vector(orc_sim* s, const double* cons, const double* prims, const double* aux, int dir) {
  double c[14], p[11], a[17], f[14];
  for (int i = 0; i < s->Nx; i++)
    for (int j = 0; j < s->Ny; j++)
      for (int k = 0; k < s->Nz; k++) {
        for (int v = 0; v < s->NC; v++) c[v] = cons[IDX(s, v, i, j, k)];
        for (int v = 0; v < s->NP; v++) p[v] = prims[IDX(s, v, i, j, k)];
        for (int v = 0; v < s->NA; v++) a[v] = aux[IDX(s, v, i, j, k)];
        if (s->NC == 9) srmhd_flux_cell(c, p, a, dir, f);
        else srrmhd_flux_cell(c, p, a, dir, f);
        for (int v = 0; v < s->NC; v++) s->f[IDX(s, v, i, j, k)] = f[v];
      }
}

static void flux_reconstruction(orc_sim* s, const double* cons, int dir, double* frecon) {
  const int shift = (s->c.weno + 1) / 2;
  size_t stride = dir == 0 ? (size_t)s->Ny * s->Nz : (dir == 1 ? (size_t)s->Nz : 1);
  size_t n = (size_t)s->NC * s->Ntot;
  for (size_t q = 0; q < n; q++) {
    s->fplus[q] = 0.5 * (s->f[q] + 1.0 * cons[q]);
    s->fminus[q] = 0.5 * (s->f[q] - 1.0 * cons[q]);
    s->fprec[q] = 0.0;
    s->fmrec[q] = 0.0;
  }
  for (int v = 0; v < s->NC; v++)
    for (int i = 0; i < s->Nx; i++)
      for (int j = 0; j < s->Ny; j++)
        for (int k = 0; k < s->Nz; k++) {
          int idx = dir == 0 ? i : (dir == 1 ? j : k);
          int N = dir == 0 ? s->Nx : (dir == 1 ? s->Ny : s->Nz);
          size_t o = IDX(s, v, i, j, k);
          const double *P = s->fplus + o, *M = s->fminus + o;
          if (idx < shift || idx >= N - shift) continue;
          {
            /* upwind cells i-shift .. i-shift+order-1, downwind i+shift-1 .. i+shift-order */
            double vu[11], vd[11];
            for (int m = 0; m < s->c.weno; m++) {
              vu[m] = P[(long)(m - shift) * (long)stride];
              vd[m] = M[(long)(shift - 1 - m) * (long)stride];
            }
            s->fprec[o] = weno_point(s->c.weno, vu);
            s->fmrec[o] = weno_point(s->c.weno, vd);
          }
        }
  for (size_t q = 0; q < n; q++) frecon[q] = s->fprec[q] + s->fmrec[q];
}

int orc_flux_F(void* h, const double* cons, const double* prims, const double* aux, double* fnet) {
  orc_sim* s = (orc_sim*)h;
  flux_vector(s, cons, prims, aux, 0);
  flux_reconstruction(s, cons, 0, s->fx);
  if (s->dims > 1) { flux_vector(s, cons, prims, aux, 1); flux_reconstruction(s, cons, 1, s->fy); }
  if (s->dims > 2) { flux_vector(s, cons, prims, aux, 2); flux_reconstruction(s, cons, 2, s->fz); }
  for (int v = 0; v < s->NC; v++)
    for (int i = s->is; i < s->ie; i++)
      for (int j = s->js; j < s->je; j++)
        for (int k = s->ks; k < s->ke; k++) {
          size_t o = IDX(s, v, i, j, k);
          if (s->dims == 3)
            fnet[o] = (s->fx[IDX(s, v, i + 1, j, k)] / s->dx - s->fx[o] / s->dx) +
                      (s->fy[IDX(s, v, i, j + 1, k)] / s->dy - s->fy[o] / s->dy) +
                      (s->fz[IDX(s, v, i, j, k + 1)] / s->dz - s->fz[o] / s->dz);
          else if (s->dims == 2)
            fnet[o] = (s->fx[IDX(s, v, i + 1, j, k)] / s->dx - s->fx[o] / s->dx) +
                      (s->fy[IDX(s, v, i, j + 1, k)] / s->dy - s->fy[o] / s->dy);
          else
            fnet[o] = (s->fx[IDX(s, v, i + 1, j, k)] / s->dx - s->fx[o] / s->dx);
        }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Model dispatch                                                            */

int orc_c2p(void* h, double* cons, double* prims, double* aux) {
  orc_sim* s = (orc_sim*)h;
  if (s->NC == 9) { srmhd_c2p(s, cons, prims, aux); return 0; }
  return srrmhd_c2p(s, cons, prims, aux);
}

/* SRMHD::solution (2 x Ntot, per cell (v^2, rho h W^2)): copied out into
 * `get` and/or replaced by `set` (either may be NULL).  Returns the number of
 * cells the last SRMHD C2P's neighbour-average retry left unconverged (the
 * reference prints these, srmhd.cc:495-498). */
int orc_srmhd_solution(void* h, double* get, const double* set) {
  orc_sim* s = (orc_sim*)h;
  if (get) memcpy(get, s->solution, (size_t)2 * s->Ntot * 8);
  if (set) memcpy(s->solution, set, (size_t)2 * s->Ntot * 8);
  return s->c2p_unconverged;
}

void orc_prims_to_all(void* h, double* cons, double* prims, double* aux) {
  orc_sim* s = (orc_sim*)h;
  if (s->NC == 9) srmhd_prims_to_all(s, cons, prims, aux);
  else srrmhd_prims_to_all(s, cons, prims, aux);
}

void orc_source(void* h, const double* cons, const double* prims, const double* aux, double* src) {
  orc_sim* s = (orc_sim*)h;
  (void)prims;
  for (int i = 0; i < s->Nx; i++)
    for (int j = 0; j < s->Ny; j++)
      for (int k = 0; k < s->Nz; k++) {
        if (s->NC == 9) {
          for (int v = 0; v < 9; v++)
            src[IDX(s, v, i, j, k)] = v == 8 ? -cons[IDX(s, 8, i, j, k)] / (s->c.cp * s->c.cp) : 0;
        } else {
          double c[14], a[17], o[14];
          for (int v = 0; v < 14; v++) c[v] = cons[IDX(s, v, i, j, k)];
          for (int v = 0; v < 17; v++) a[v] = aux[IDX(s, v, i, j, k)];
          srrmhd_source_cell(c, a, s->c.cp, o);
          for (int v = 0; v < 14; v++) src[IDX(s, v, i, j, k)] = o[v];
        }
      }
}

/* TimeIntegrator::finalise (timeInt.h:117-132) */
static int finalise(orc_sim* s, double* cons, double* prims, double* aux) {
  int rc = orc_c2p(s, cons, prims, aux);
  orc_apply_bcs(s, cons, prims, aux);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Integrators                                                               */

static int rk2_step(orc_sim* s, double dt) {
  size_t nI;
  (void)nI;
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) {
        for (int v = 0; v < s->NA; v++) s->p1aux[IDX(s, v, i, j, k)] = s->aux[IDX(s, v, i, j, k)];
        for (int v = 0; v < s->NP; v++) s->p1prims[IDX(s, v, i, j, k)] = s->prims[IDX(s, v, i, j, k)];
      }
  orc_flux_F(s, s->cons, s->prims, s->aux, s->args1);
  for (int v = 0; v < s->NC; v++)
    for (int i = s->is; i < s->ie; i++)
      for (int j = s->js; j < s->je; j++)
        for (int k = s->ks; k < s->ke; k++) {
          size_t o = IDX(s, v, i, j, k);
          s->p1cons[o] = s->cons[o] - dt * s->args1[o];
        }
  if (finalise(s, s->p1cons, s->p1prims, s->p1aux)) return 1;
  orc_flux_F(s, s->p1cons, s->p1prims, s->p1aux, s->args2);
  for (int v = 0; v < s->NC; v++)
    for (int i = s->is; i < s->ie; i++)
      for (int j = s->js; j < s->je; j++)
        for (int k = s->ks; k < s->ke; k++) {
          size_t o = IDX(s, v, i, j, k);
          s->cons[o] = 0.5 * (s->cons[o] + s->p1cons[o] - dt * s->args2[o]);
        }
  return finalise(s, s->cons, s->prims, s->aux);
}

static int rksplit_step(orc_sim* s, double dt) {
  if (rk2_step(s, dt)) return 1;
  orc_source(s, s->cons, s->prims, s->aux, s->source);
  for (int v = 0; v < s->NC; v++)
    for (int i = s->is; i < s->ie; i++)
      for (int j = s->js; j < s->je; j++)
        for (int k = s->ks; k < s->ke; k++) {
          size_t o = IDX(s, v, i, j, k);
          s->cons[o] += dt * s->source[o];
        }
  return finalise(s, s->cons, s->prims, s->aux);
}

/* IMEX residuals.  kind 1, 2: SSP2(222) stages 1, 2 (SSP2.cc:194-264), also
 * SSP3(332) stages 1, 2 (SSP3.cc:237-314, the same expressions); kind 3:
 * SSP3(332) stage 3 (SSP3.cc:335-355); kinds 4, 5, 6: SSP2(322) stages 1-3
 * (SSP2322.cc:262-383). */
typedef struct {
  double cons[14], aux10, flux1[14], source1[14], flux2[14], source2[14], dt, g, sigma, cp;
  int stage;
  const orc_config* cfg; /* for a functional conductivity */
} imex_ctx;

static void imex_residual(void* ctx, int n, const double* x, double* fvec) {
  imex_ctx* a = (imex_ctx*)ctx;
  /* SSP2's constructor assigns IMEX2Arguments(data), but the assignment
   * operator (IMEX2Args.cc:34-63) does not copy gam / om2gam, so the values in
   * effect are the default constructor's (IMEX2Args.h:35-37). */
  const double gam = 0.2928932188134525, om2gam = 0.4142135623730950;
  double p[11], ax[17], src[14];
  ax[10] = a->aux10;
  int ok = srrmhd_c2p_cell(x, a->g, sigma_func(a->cfg, x[0]), p, ax);
  a->aux10 = ax[10];
  if (!ok) { for (int i = 0; i < n; i++) fvec[i] = 1.0e6; return; }
  srrmhd_source_cell(x, ax, a->cp, src);
  /* IMEX3Arguments (IMEX3Args.h:28-29) adds hmgam; SSP3's assignment from
   * IMEX3Arguments(data) keeps the default-constructed constants as well. */
  const double hmgam = 0.2071067811865475;
  switch (a->stage) {
    case 1:
      for (int i = 0; i < n; i++) fvec[i] = x[i] - a->cons[i] - a->dt * gam * src[i];
      break;
    case 2:
      for (int i = 0; i < n; i++)
        fvec[i] = x[i] - a->cons[i] + a->dt * (a->flux1[i] - om2gam * a->source1[i] - gam * src[i]);
      break;
    case 3:
      for (int i = 0; i < n; i++)
        fvec[i] = x[i] - a->cons[i] + a->dt * (a->flux1[i] + a->flux2[i]) / 4.0 -
                  a->dt * (hmgam * a->source1[i] + gam * src[i]);
      break;
    case 4:
      for (int i = 0; i < n; i++) fvec[i] = x[i] - a->cons[i] - a->dt * 0.5 * src[i];
      break;
    case 5:
      for (int i = 0; i < n; i++)
        fvec[i] = x[i] - a->cons[i] + a->dt * 0.5 * (a->source1[i] - src[i]);
      break;
    default:
      for (int i = 0; i < n; i++)
        fvec[i] = x[i] - a->cons[i] + a->dt * (a->flux2[i] - 0.5 * a->source2[i] - 0.5 * src[i]);
      break;
  }
}

/* One implicit stage of SSP3 / SSP2322 over the interior: initial guess x0
 * (xform 0: U^n; 1: U1; 2: U2 + dt (F1 + F2) / 4; 3: (U^n + U2 - dt F2) / 2),
 * Z guess from zaux[10]; writes U_k and, as the reference copies args.aux
 * back to tempaux, the last evaluation's Z into taux[10]. */
static int imex_stage_sweep(orc_sim* s, int kind, int xform, double dt, double tol,
                            const double* zaux, double* out) {
  imex_ctx ctx;
  double x[14], fvec[14];
  ctx.dt = dt; ctx.g = s->c.gamma; ctx.sigma = s->c.sigma; ctx.cp = s->c.cp; ctx.cfg = &s->c;
  ctx.stage = kind;
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) {
        for (int v = 0; v < 14; v++) {
          size_t o = IDX(s, v, i, j, k);
          ctx.cons[v] = s->cons[o];
          ctx.flux1[v] = s->flux1[o];
          ctx.source1[v] = s->source1[o];
          ctx.flux2[v] = s->flux2[o];
          ctx.source2[v] = s->source2[o];
          if (xform == 0) x[v] = s->cons[o];
          else if (xform == 1) x[v] = s->U1[o];
          else if (xform == 2) x[v] = s->U2[o] + dt * (s->flux1[o] + s->flux2[o]) / 4.0;
          else x[v] = 0.5 * (s->cons[o] + s->U2[o] - dt * s->flux2[o]);
        }
        ctx.aux10 = zaux[IDX(s, 10, i, j, k)];
        if (orc_hybrd1(imex_residual, &ctx, 14, x, fvec, tol, NULL) != 1) return 2;
        for (int v = 0; v < 14; v++) out[IDX(s, v, i, j, k)] = x[v];
        s->taux[IDX(s, 10, i, j, k)] = ctx.aux10;
      }
  return 0;
}

/* SSP3::step (SSP3.cc:43-216) */
static int ssp3_step(orc_sim* s, double dt) {
  const double tol = 0.0000000149011612;
  int rc;
  if ((rc = imex_stage_sweep(s, 1, 0, dt, tol, s->aux, s->U1))) return rc;
  if (finalise(s, s->U1, s->tprims, s->taux)) return 1;
  orc_source(s, s->U1, s->tprims, s->taux, s->source1);
  orc_flux_F(s, s->U1, s->tprims, s->taux, s->flux1);
  if ((rc = imex_stage_sweep(s, 2, 1, dt, tol, s->taux, s->U2))) return rc;
  if (finalise(s, s->U2, s->tprims, s->taux)) return 1;
  orc_source(s, s->U2, s->tprims, s->taux, s->source2);
  orc_flux_F(s, s->U2, s->tprims, s->taux, s->flux2);
  /* stage 3 starts from the step's own prims / aux (SSP3.cc:146-159) */
  if ((rc = imex_stage_sweep(s, 3, 2, dt, tol, s->aux, s->U3))) return rc;
  if (finalise(s, s->U3, s->tprims, s->taux)) return 1;
  orc_source(s, s->U3, s->tprims, s->taux, s->source3);
  orc_flux_F(s, s->U3, s->tprims, s->taux, s->flux3);
  for (int v = 0; v < 14; v++)
    for (int i = s->is; i < s->ie; i++)
      for (int j = s->js; j < s->je; j++)
        for (int k = s->ks; k < s->ke; k++) {
          size_t o = IDX(s, v, i, j, k);
          s->cons[o] = s->cons[o] - dt * (s->flux1[o] + s->flux2[o] + 4 * s->flux3[o]) / 6.0 +
                       dt * (s->source1[o] + s->source2[o] + 4 * s->source3[o]) / 6.0;
        }
  return finalise(s, s->cons, s->prims, s->aux);
}

/* SSP2322::step (SSP2322.cc:68-249).  F(U1) is computed there but never
 * used, so it is skipped. */
static int ssp2322_step(orc_sim* s, double dt) {
  const double tol = 1.48e-8;
  int rc;
  if ((rc = imex_stage_sweep(s, 4, 0, dt, tol, s->aux, s->U1))) return rc;
  if (finalise(s, s->U1, s->tprims, s->taux)) return 1;
  orc_source(s, s->U1, s->tprims, s->taux, s->source1);
  if ((rc = imex_stage_sweep(s, 5, 0, dt, tol, s->aux, s->U2))) return rc;
  if (finalise(s, s->U2, s->tprims, s->taux)) return 1;
  orc_source(s, s->U2, s->tprims, s->taux, s->source2);
  orc_flux_F(s, s->U2, s->tprims, s->taux, s->flux2);
  if ((rc = imex_stage_sweep(s, 6, 3, dt, tol, s->aux, s->U3))) return rc;
  if (finalise(s, s->U3, s->tprims, s->taux)) return 1;
  orc_source(s, s->U3, s->tprims, s->taux, s->source3);
  orc_flux_F(s, s->U3, s->tprims, s->taux, s->flux3);
  for (int v = 0; v < 14; v++)
    for (int i = s->is; i < s->ie; i++)
      for (int j = s->js; j < s->je; j++)
        for (int k = s->ks; k < s->ke; k++) {
          size_t o = IDX(s, v, i, j, k);
          s->cons[o] = s->cons[o] - dt * 0.5 * (s->flux2[o] + s->flux3[o] - s->source2[o] -
                                                s->source3[o]);
        }
  /* prims / aux take U3's finalised values (SSP2322.cc:236-245): only aux[10]
   * seeds the final recovery */
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) {
        for (int v = 0; v < s->NP; v++) s->prims[IDX(s, v, i, j, k)] = s->tprims[IDX(s, v, i, j, k)];
        for (int v = 0; v < s->NA; v++) s->aux[IDX(s, v, i, j, k)] = s->taux[IDX(s, v, i, j, k)];
      }
  return finalise(s, s->cons, s->prims, s->aux);
}

static int ssp2_step(orc_sim* s, double dt) {
  const double tol = 0.000000149011612;
  imex_ctx ctx;
  double x[14], fvec[14];
  ctx.dt = dt; ctx.g = s->c.gamma; ctx.sigma = s->c.sigma; ctx.cp = s->c.cp; ctx.cfg = &s->c;
  ctx.stage = 1;
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) {
        for (int v = 0; v < 14; v++) x[v] = ctx.cons[v] = s->cons[IDX(s, v, i, j, k)];
        ctx.aux10 = s->aux[IDX(s, 10, i, j, k)];
        if (orc_hybrd1(imex_residual, &ctx, 14, x, fvec, tol, NULL) != 1) return 2;
        for (int v = 0; v < 14; v++) s->U1[IDX(s, v, i, j, k)] = x[v];
      }
  if (finalise(s, s->U1, s->prims, s->aux)) return 1;
  orc_source(s, s->U1, s->prims, s->aux, s->source1);
  orc_flux_F(s, s->U1, s->prims, s->aux, s->flux1);
  ctx.stage = 2;
  for (int i = s->is; i < s->ie; i++)
    for (int j = s->js; j < s->je; j++)
      for (int k = s->ks; k < s->ke; k++) {
        for (int v = 0; v < 14; v++) {
          size_t o = IDX(s, v, i, j, k);
          ctx.cons[v] = s->cons[o];
          ctx.flux1[v] = s->flux1[o];
          ctx.source1[v] = s->source1[o];
          x[v] = 0.5 * (s->cons[o] + s->U1[o] - dt * s->flux1[o]);
        }
        ctx.aux10 = s->aux[IDX(s, 10, i, j, k)];
        if (orc_hybrd1(imex_residual, &ctx, 14, x, fvec, tol, NULL) != 1) return 2;
        for (int v = 0; v < 14; v++) s->U2[IDX(s, v, i, j, k)] = x[v];
      }
  if (finalise(s, s->U2, s->prims, s->aux)) return 1;
  orc_source(s, s->U2, s->prims, s->aux, s->source2);
  orc_flux_F(s, s->U2, s->prims, s->aux, s->flux2);
  for (int v = 0; v < 14; v++)
    for (int i = s->is; i < s->ie; i++)
      for (int j = s->js; j < s->je; j++)
        for (int k = s->ks; k < s->ke; k++) {
          size_t o = IDX(s, v, i, j, k);
          s->cons[o] += -0.5 * dt * (s->flux1[o] + s->flux2[o] - s->source1[o] - s->source2[o]);
        }
  return finalise(s, s->cons, s->prims, s->aux);
}

/* ------------------------------------------------------------------------ */
/* Simulation                                                                */

void orc_destroy(void* h) {
  orc_sim* s = (orc_sim*)h;
  if (!s) return;
  double* arrs[] = {s->cons, s->prims, s->aux, s->f, s->p1cons, s->p1prims, s->p1aux, s->args1,
                    s->args2, s->U1, s->U2, s->flux1, s->flux2, s->source1, s->source2,
                    s->solution, s->fplus, s->fminus, s->fprec, s->fmrec, s->fx, s->fy, s->fz,
                    s->source, s->U3, s->flux3, s->source3, s->tprims, s->taux};
  for (size_t q = 0; q < sizeof arrs / sizeof arrs[0]; q++) free(arrs[q]);
  free(s);
}

void* orc_create(const orc_config* c, const double* prims) {
  orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
  double zmin = c->zmin, zmax = c->zmax, ymin = c->ymin, ymax = c->ymax;
  s->c = *c;
  s->NC = c->model == 0 ? 9 : 14;
  s->NP = c->model == 0 ? 8 : 11;
  s->NA = c->model == 0 ? 13 : 17;
  s->Nx = c->nx + 2 * c->Ng;
  s->Ny = c->ny + 2 * c->Ng;
  s->Nz = c->nz + 2 * c->Ng;
  s->dims = 3;
  if (c->nz == 0) { s->Nz = 1; zmin = -1e20; zmax = 1e20; s->dims = 2; }
  if (c->ny == 0) { s->Nz = s->Ny = 1; zmin = ymin = -1e20; zmax = ymax = 1e20; s->dims = 1; }
  s->Ntot = s->Nx * s->Ny * s->Nz;
  s->is = c->Ng; s->ie = s->Nx - c->Ng;
  s->js = c->Ng; s->je = s->Ny - c->Ng;
  s->ks = c->Ng; s->ke = s->Nz - c->Ng;
  if (s->dims < 3) { s->ks = 0; s->ke = 1; }
  if (s->dims < 2) { s->js = 0; s->je = 1; }
  if (c->sigma < 0.0 || c->Ng < (c->weno + 1) / 2 + 1 ||
      (c->weno != 3 && c->weno != 5 && c->weno != 7 && c->weno != 9 && c->weno != 11)) {
    free(s);
    return NULL;
  }
  s->dx = (c->xmax - c->xmin) / (c->nx);
  s->dy = (ymax - ymin) / (c->ny);
  s->dz = (zmax - zmin) / (c->nz);
  size_t nc = (size_t)s->NC * s->Ntot, np = (size_t)s->NP * s->Ntot, na = (size_t)s->NA * s->Ntot;
  s->cons = (double*)calloc(nc, 8); s->prims = (double*)calloc(np, 8); s->aux = (double*)calloc(na, 8);
  s->f = (double*)calloc(nc, 8); s->source = (double*)calloc(nc, 8);
  s->p1cons = (double*)calloc(nc, 8); s->p1prims = (double*)calloc(np, 8); s->p1aux = (double*)calloc(na, 8);
  s->args1 = (double*)calloc(nc, 8); s->args2 = (double*)calloc(nc, 8);
  s->U1 = (double*)calloc(nc, 8); s->U2 = (double*)calloc(nc, 8);
  s->flux1 = (double*)calloc(nc, 8); s->flux2 = (double*)calloc(nc, 8);
  s->source1 = (double*)calloc(nc, 8); s->source2 = (double*)calloc(nc, 8);
  s->U3 = (double*)calloc(nc, 8); s->flux3 = (double*)calloc(nc, 8);
  s->source3 = (double*)calloc(nc, 8);
  s->tprims = (double*)calloc(np, 8); s->taux = (double*)calloc(na, 8);
  s->solution = (double*)calloc((size_t)2 * s->Ntot, 8);
  s->fplus = (double*)calloc(nc, 8); s->fminus = (double*)calloc(nc, 8);
  s->fprec = (double*)calloc(nc, 8); s->fmrec = (double*)calloc(nc, 8);
  s->fx = (double*)calloc(nc, 8); s->fy = (double*)calloc(nc, 8); s->fz = (double*)calloc(nc, 8);
  memcpy(s->prims, prims, np * 8);
  orc_prims_to_all(s, s->cons, s->prims, s->aux);
  orc_apply_bcs(s, s->cons, s->prims, s->aux);
  {
    double dtX = c->cfl * s->dx / (1.0 * sqrt(s->dims));
    double dtY = c->cfl * s->dy / (1.0 * sqrt(s->dims));
    double dtZ = c->cfl * s->dz / (1.0 * sqrt(s->dims));
    s->dt = (dtX < dtY && dtX < dtZ) ? dtX : ((dtY < dtZ) ? dtY : dtZ);
  }
  return s;
}

int orc_step(void* h, double dt) {
  orc_sim* s = (orc_sim*)h;
  if (s->c.integrator == 0) return rk2_step(s, dt);
  if (s->c.integrator == 1) return rksplit_step(s, dt);
  if (s->c.integrator == 3) return ssp3_step(s, dt);
  if (s->c.integrator == 4) return ssp2322_step(s, dt);
  return ssp2_step(s, dt);
}

/* Simulation::updateTime (simulation.cc:104-133) */
int orc_update_time(void* h, int n) {
  orc_sim* s = (orc_sim*)h;
  for (int q = 0; q < n; q++) {
    double dtX = s->c.cfl * s->dx / (1.0 * sqrt(s->dims));
    double dtY = s->c.cfl * s->dy / (1.0 * sqrt(s->dims));
    double dtZ = s->c.cfl * s->dz / (1.0 * sqrt(s->dims));
    int rc;
    s->dt = (dtX <= dtY && dtX <= dtZ) ? dtX : ((dtY < dtZ) ? dtY : dtZ);
    if (s->iters < 15) s->dt *= 0.1;
    if (s->iters >= 15 && s->iters < 30) s->dt *= 0.25;
    if (s->t + s->dt > s->c.endTime) s->dt = s->c.endTime - s->t;
    rc = orc_step(s, s->dt);
    if (rc) return rc;
    s->t += s->dt;
    s->iters++;
  }
  return 0;
}

void orc_info(void* h, int* ints, double* dbls) {
  orc_sim* s = (orc_sim*)h;
  ints[0] = s->Nx; ints[1] = s->Ny; ints[2] = s->Nz;
  ints[3] = s->NC; ints[4] = s->NP; ints[5] = s->NA;
  ints[6] = s->iters; ints[7] = s->dims;
  dbls[0] = s->t; dbls[1] = s->dt; dbls[2] = s->dx; dbls[3] = s->dy; dbls[4] = s->dz;
}

void orc_get_state(void* h, double* cons, double* prims, double* aux) {
  orc_sim* s = (orc_sim*)h;
  if (cons) memcpy(cons, s->cons, (size_t)s->NC * s->Ntot * 8);
  if (prims) memcpy(prims, s->prims, (size_t)s->NP * s->Ntot * 8);
  if (aux) memcpy(aux, s->aux, (size_t)s->NA * s->Ntot * 8);
}

void orc_set_state(void* h, const double* cons, const double* prims, const double* aux) {
  orc_sim* s = (orc_sim*)h;
  if (cons) memcpy(s->cons, cons, (size_t)s->NC * s->Ntot * 8);
  if (prims) memcpy(s->prims, prims, (size_t)s->NP * s->Ntot * 8);
  if (aux) memcpy(s->aux, aux, (size_t)s->NA * s->Ntot * 8);
}

/* Per-cell SRMHD primitive recovery from a (v^2, rho h W^2) guess: one
 * hybrd1 solve per cell at tolerance tol (the grid C2P uses 1.49011612e-7,
 * srmhd.cc:380; the single-cell C2P 1.4e-8, srmhd.cc:308). */
int orc_srmhd_c2p_cells(int n, double gamma, double tol, const double* cons, const double* guess,
                        double* sol, int* info, int* nfev) {
  int bad = 0;
  for (int q = 0; q < n; q++) {
    const double* c = cons + 9 * q;
    srmhd_args a;
    double x[2] = {guess[2 * q], guess[2 * q + 1]}, r[2];
    a.D = c[0]; a.g = gamma; a.tau = c[4];
    a.BS = c[5] * c[1] + c[6] * c[2] + c[7] * c[3];
    a.Bsq = c[5] * c[5] + c[6] * c[6] + c[7] * c[7];
    a.Ssq = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
    info[q] = orc_hybrd1(srmhd_residual, &a, 2, x, r, tol, &nfev[q]);
    if (info[q] != 1) bad++;
    sol[2 * q] = x[0];
    sol[2 * q + 1] = x[1];
  }
  return bad;
}
#undef C
#undef P
#undef A
#undef SOL
