// Device Powell-hybrid root finder with the iterates of the reference's
// vendored MINPACK `hybrd1` (Project/CPU/CminpackLibrary/Src/hybrd1.cc:114-143,
// hybrd.cc:213-575, fdjac1.cc, qrfac.cc, qform.cc, dogleg.cc, r1updt.cc,
// r1mpyq.cc, enorm.cc).
//
// The algorithm is MINPACK's published hybrid method (More, Garbow, Hillstrom,
// Argonne 1980): forward-difference Jacobian, Householder QR without pivoting,
// dogleg step inside a trust region, Broyden rank-one updates of Q and R, a
// new Jacobian after two failed steps.  It is written here from scratch for
// one thread per system with N a compile-time constant, so that for N = 2
// every array lives in registers.  Three properties of the reference build are
// kept on purpose because the iterates depend on them:
//   * hybrd1 settings: diag = 1 (mode 2), factor = 100, maxfev = 200 (N + 1),
//     ml = mu = N - 1 (dense Jacobian), info 5 reported as 4;
//   * the vendored edits: machine epsilon for the xtol-too-small test is
//     xtol^2 (hybrd.cc:222-223) and the difference step is the fixed
//     1.414213562373095e-08 * |x_j|, replaced by that constant below 1e-17
//     (fdjac1.cc);
//   * every sum is accumulated in the reference's order, starting from +0.
// With diag identically one the reference's multiplications and divisions by
// diag are exact and are omitted.
// Matrices are column-major, a(i, j) = a[i + N*j]; R is the packed upper
// triangle stored by rows, R(i, j) at rpos(i, j).
#pragma once
#include <cfloat>

namespace mth {

struct HybrdResult {
  int info;  // 1 converged, 2 maxfev, 3 xtol too small, 4 slow progress, 0 bad input
  int nfev;
};

// Euclidean norm with MINPACK's three-range accumulation (enorm.cc), the
// dwarf / giant limits of the reference's double build.
template <int M>
__device__ __forceinline__ double hy_enorm_ranges(const double* x) {
  const double rdwarf = 1.82691291192569e-153;
  const double rgiant = 1.34078079299426e+153;
  double s1 = 0., s2 = 0., s3 = 0., x1max = 0., x3max = 0.;
  const double agiant = rgiant / (double)M;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    double xabs = fabs(x[i]);
    if (xabs >= agiant) {
      if (xabs > x1max) {
        double d1 = x1max / xabs;
        s1 = 1. + s1 * (d1 * d1);
        x1max = xabs;
      } else {
        double d1 = xabs / x1max;
        s1 += d1 * d1;
      }
    } else if (xabs <= rdwarf) {
      if (xabs > x3max) {
        double d1 = x3max / xabs;
        s3 = 1. + s3 * (d1 * d1);
        x3max = xabs;
      } else if (xabs != 0.) {
        double d1 = xabs / x3max;
        s3 += d1 * d1;
      }
    } else {
      s2 += xabs * xabs;
    }
  }
  if (s1 != 0.) return x1max * sqrt(s1 + (s2 / x1max) / x1max);
  if (s2 != 0.) {
    if (s2 >= x3max) return sqrt(s2 * (1. + (x3max / s2) * (x3max * s3)));
    return sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
  }
  return x3max * sqrt(s3);
}

// enorm's arguments by value, so that its out-of-line form keeps the
// caller's vector in registers.
template <int M>
struct EnormArgs {
  double x[M];
};

template <int M>
__device__ __noinline__ double hy_enorm_full(EnormArgs<M> a) {
  return hy_enorm_ranges<M>(a.x);
}

// enorm for the usual vector, every component zero or of intermediate size
// (rdwarf < |x| < rgiant / M): the three-range accumulation then adds only
// to s2, in index order from zero, and returns
// sqrt(s2 * (1 + (0 / s2) * (0 * s3))) = sqrt(s2), or x3max * sqrt(s3) = 0
// when every component is zero, which sqrt(s2) also gives.  Any other vector
// takes the full form, out of line: the many call sites of the hybrid
// method then carry the short form only.
template <int M>
__device__ __forceinline__ double hy_enorm(const double* x) {
  const double rdwarf = 1.82691291192569e-153;
  const double agiant = 1.34078079299426e+153 / (double)M;
  double s2 = 0.;
  bool mid = true;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const double xabs = fabs(x[i]);
    mid = mid && xabs < agiant && (xabs > rdwarf || xabs == 0.);
    s2 += xabs * xabs;
  }
  if (mid) return sqrt(s2);
  EnormArgs<M> a;
#pragma unroll
  for (int i = 0; i < M; ++i) a.x[i] = x[i];
  return hy_enorm_full<M>(a);
}

template <int N>
struct Hybrd {
  // Loops are unrolled by an explicit factor of 16: loops with a constant trip
  // count (at most N) unroll completely, and so do the triangular loops whose
  // bounds depend on an outer index, which a bare "#pragma unroll" leaves
  // rolled.  Order of operations is unchanged.  14-unknown implicit stages:
  // 4.54 -> 3.77 ms per SSP2 step at 256x512 (factors 4 and 8 are slower).
  static constexpr int UNR = 16;
  static constexpr int LR = N * (N + 1) / 2;
  __device__ static constexpr int rpos(int i, int j) { return i * N - i * (i - 1) / 2 + (j - i); }

  // Givens pair used by r1updt: from (a, b) with |a| the "pivot" entry.
  __device__ static __forceinline__ void givens(double num, double den, bool swap, double& c,
                                                double& s, double& tau) {
    const double giant = DBL_MAX;
    if (swap) {  // |den| < |num| branch of r1updt: cotan = den / num
      double cotan = den / num;
      s = .5 / sqrt(.25 + .25 * (cotan * cotan));
      c = s * cotan;
      tau = 1.;
      if (fabs(c) * giant > 1.) tau = 1. / c;
    } else {
      double tn = num / den;
      c = .5 / sqrt(.25 + .25 * (tn * tn));
      s = c * tn;
      tau = s;
    }
  }

  // Recovers (cos, sin) from the stored tau of a Givens rotation (r1mpyq.cc).
  __device__ static __forceinline__ void unpack(double t, double& c, double& s) {
    if (fabs(t) > 1.) {
      c = 1. / t;
      s = sqrt(1. - c * c);
    } else {
      s = t;
      c = sqrt(1. - s * s);
    }
  }

  template <class F>
  __device__ static HybrdResult solve(F& fcn, double* x, double* fvec, double xtol) {
    const int maxfev = 200 * (N + 1);
    const double epsmch = xtol * xtol;
    const double factor = 100.;
    double fjac[N * N], r[LR], qtf[N], wa1[N], wa2[N], wa3[N], wa4[N];
    HybrdResult res{0, 0};
    if (xtol < 0.) return res;

    fcn(x, fvec);
    int nfev = 1;
    double fnorm = hy_enorm<N>(fvec);
    int iter = 1, ncsuc = 0, ncfail = 0, nslow1 = 0, nslow2 = 0;
    double delta = 0., xnorm = 0.;
    int info = 0;

    for (;;) {
      bool jeval = true;
      // Forward-difference Jacobian, one column per shifted evaluation.
      const double eps = 1.414213562373095e-08;
      for (int j = 0; j < N; ++j) {
        double temp = x[j];
        double h = eps * fabs(temp);
        if (h < 1.0e-17) h = eps;
        x[j] = temp + h;
        fcn(x, wa1);
        x[j] = temp;
#pragma unroll (UNR)
        for (int i = 0; i < N; ++i) fjac[i + N * j] = (wa1[i] - fvec[i]) / h;
      }
      nfev += N;

      // Householder QR of fjac (no pivoting): wa1 = rdiag.
#pragma unroll (UNR)
      for (int j = 0; j < N; ++j) {
        double ajnorm = hy_enorm_tail(fjac + j + N * j, N - j);
        if (ajnorm != 0.) {
          if (fjac[j + N * j] < 0.) ajnorm = -ajnorm;
#pragma unroll (UNR)
          for (int i = j; i < N; ++i) fjac[i + N * j] /= ajnorm;
          fjac[j + N * j] += 1.;
#pragma unroll (UNR)
          for (int k = j + 1; k < N; ++k) {
            double sum = 0.;
#pragma unroll (UNR)
            for (int i = j; i < N; ++i) sum += fjac[i + N * j] * fjac[i + N * k];
            double temp = sum / fjac[j + N * j];
#pragma unroll (UNR)
            for (int i = j; i < N; ++i) fjac[i + N * k] -= temp * fjac[i + N * j];
          }
        }
        wa1[j] = -ajnorm;
      }

      if (iter == 1) {
#pragma unroll (UNR)
        for (int j = 0; j < N; ++j) wa3[j] = x[j];
        xnorm = hy_enorm<N>(wa3);
        delta = factor * xnorm;
        if (delta == 0.) delta = factor;
      }

      // qtf = Q^T fvec from the Householder vectors.
#pragma unroll (UNR)
      for (int i = 0; i < N; ++i) qtf[i] = fvec[i];
#pragma unroll (UNR)
      for (int j = 0; j < N; ++j) {
        if (fjac[j + N * j] != 0.) {
          double sum = 0.;
#pragma unroll (UNR)
          for (int i = j; i < N; ++i) sum += fjac[i + N * j] * qtf[i];
          double temp = -sum / fjac[j + N * j];
#pragma unroll (UNR)
          for (int i = j; i < N; ++i) qtf[i] += fjac[i + N * j] * temp;
        }
      }

      // R from the strict upper triangle and rdiag.
#pragma unroll (UNR)
      for (int j = 0; j < N; ++j) {
#pragma unroll (UNR)
        for (int i = 0; i < j; ++i) r[rpos(i, j)] = fjac[i + N * j];
        r[rpos(j, j)] = wa1[j];
      }

      // Accumulate Q in fjac (qform.cc with m = n).
#pragma unroll (UNR)
      for (int j = 1; j < N; ++j) {
#pragma unroll (UNR)
        for (int i = 0; i < j; ++i) fjac[i + N * j] = 0.;
      }
#pragma unroll (UNR)
      for (int l = 0; l < N; ++l) {
        const int k = N - 1 - l;
#pragma unroll (UNR)
        for (int i = k; i < N; ++i) {
          wa1[i] = fjac[i + N * k];
          fjac[i + N * k] = 0.;
        }
        fjac[k + N * k] = 1.;
        if (wa1[k] != 0.) {
#pragma unroll (UNR)
          for (int j = k; j < N; ++j) {
            double sum = 0.;
#pragma unroll (UNR)
            for (int i = k; i < N; ++i) sum += fjac[i + N * j] * wa1[i];
            double temp = sum / wa1[k];
#pragma unroll (UNR)
            for (int i = k; i < N; ++i) fjac[i + N * j] -= temp * wa1[i];
          }
        }
      }

      // Inner loop: dogleg steps with rank-one updates.
      for (;;) {
        dogleg(r, qtf, delta, wa1, wa2, wa3);
#pragma unroll (UNR)
        for (int j = 0; j < N; ++j) {
          wa1[j] = -wa1[j];
          wa2[j] = x[j] + wa1[j];
          wa3[j] = wa1[j];
        }
        double pnorm = hy_enorm<N>(wa3);
        if (iter == 1) delta = (delta <= pnorm) ? delta : pnorm;

        fcn(wa2, wa4);
        ++nfev;
        double fnorm1 = hy_enorm<N>(wa4);

        double actred = -1.;
        if (fnorm1 < fnorm) {
          double d1 = fnorm1 / fnorm;
          actred = 1. - d1 * d1;
        }
#pragma unroll (UNR)
        for (int i = 0; i < N; ++i) {
          double sum = 0.;
#pragma unroll (UNR)
          for (int j = i; j < N; ++j) sum += r[rpos(i, j)] * wa1[j];
          wa3[i] = qtf[i] + sum;
        }
        double temp = hy_enorm<N>(wa3);
        double prered = 0.;
        if (temp < fnorm) {
          double d1 = temp / fnorm;
          prered = 1. - d1 * d1;
        }
        double ratio = 0.;
        if (prered > 0.) ratio = actred / prered;

        if (ratio < .1) {
          ncsuc = 0;
          ++ncfail;
          delta = .5 * delta;
        } else {
          ncfail = 0;
          ++ncsuc;
          if (ratio >= .5 || ncsuc > 1) {
            double d1 = pnorm / .5;
            delta = (delta >= d1) ? delta : d1;
          }
          if (fabs(ratio - 1.) <= .1) delta = pnorm / .5;
        }

        if (ratio >= 1e-4) {
#pragma unroll (UNR)
          for (int j = 0; j < N; ++j) {
            x[j] = wa2[j];
            wa2[j] = x[j];
            fvec[j] = wa4[j];
          }
          xnorm = hy_enorm<N>(wa2);
          fnorm = fnorm1;
          ++iter;
        }

        ++nslow1;
        if (actred >= .001) nslow1 = 0;
        if (jeval) ++nslow2;
        if (actred >= .1) nslow2 = 0;

        if (delta <= xtol * xnorm || fnorm == 0.) info = 1;
        if (info != 0) break;
        if (nfev >= maxfev) info = 2;
        {
          double d1 = .1 * delta;
          double m = (d1 >= pnorm) ? d1 : pnorm;
          if (.1 * m <= epsmch * xnorm) info = 3;
        }
        if (nslow2 == 5) info = 4;
        if (nslow1 == 10) info = 5;
        if (info != 0) break;
        if (ncfail == 2) break;

        // Broyden update of Q and R.
#pragma unroll (UNR)
        for (int j = 0; j < N; ++j) {
          double sum = 0.;
#pragma unroll (UNR)
          for (int i = 0; i < N; ++i) sum += fjac[i + N * j] * wa4[i];
          wa2[j] = (sum - wa3[j]) / pnorm;
          wa1[j] = (wa1[j] / pnorm);
          if (ratio >= 1e-4) qtf[j] = sum;
        }
        r1updt(r, wa1, wa2, wa3);
        r1mpyq_cols(fjac, wa2, wa3);
        r1mpyq_row(qtf, wa2, wa3);
        jeval = false;
      }
      if (info != 0) break;
    }
    res.info = (info == 5) ? 4 : info;
    res.nfev = nfev;
    return res;
  }

  // enorm over a column tail of run-time length m (used by the QR; the
  // giant threshold depends on m exactly as in the reference call).
  __device__ static __forceinline__ double hy_enorm_tail(const double* x, int m) {
    double buf[N];
#pragma unroll (UNR)
    for (int i = 0; i < N; ++i) buf[i] = (i < m) ? x[i] : 0.;
    return enorm_len(buf, m);
  }

  __device__ static __noinline__ double enorm_len_full(EnormArgs<N> a, int m) {
    return enorm_len_ranges(a.x, m);
  }

  // enorm of x[0 .. m): the short form of hy_enorm for the usual vector.
  __device__ static __forceinline__ double enorm_len(const double* x, int m) {
    const double rdwarf = 1.82691291192569e-153;
    const double agiant = 1.34078079299426e+153 / (double)m;
    double s2 = 0.;
    bool mid = true;
#pragma unroll (UNR)
    for (int i = 0; i < N; ++i) {
      if (i >= m) break;
      const double xabs = fabs(x[i]);
      mid = mid && xabs < agiant && (xabs > rdwarf || xabs == 0.);
      s2 += xabs * xabs;
    }
    if (mid) return sqrt(s2);
    EnormArgs<N> a;
#pragma unroll (UNR)
    for (int i = 0; i < N; ++i) a.x[i] = x[i];
    return enorm_len_full(a, m);
  }

  __device__ static __forceinline__ double enorm_len_ranges(const double* x, int m) {
    const double rdwarf = 1.82691291192569e-153;
    const double rgiant = 1.34078079299426e+153;
    double s1 = 0., s2 = 0., s3 = 0., x1max = 0., x3max = 0.;
    const double agiant = rgiant / (double)m;
#pragma unroll (UNR)
    for (int i = 0; i < N; ++i) {
      if (i >= m) break;
      double xabs = fabs(x[i]);
      if (xabs >= agiant) {
        if (xabs > x1max) {
          double d1 = x1max / xabs;
          s1 = 1. + s1 * (d1 * d1);
          x1max = xabs;
        } else {
          double d1 = xabs / x1max;
          s1 += d1 * d1;
        }
      } else if (xabs <= rdwarf) {
        if (xabs > x3max) {
          double d1 = x3max / xabs;
          s3 = 1. + s3 * (d1 * d1);
          x3max = xabs;
        } else if (xabs != 0.) {
          double d1 = xabs / x3max;
          s3 += d1 * d1;
        }
      } else {
        s2 += xabs * xabs;
      }
    }
    if (s1 != 0.) return x1max * sqrt(s1 + (s2 / x1max) / x1max);
    if (s2 != 0.) {
      if (s2 >= x3max) return sqrt(s2 * (1. + (x3max / s2) * (x3max * s3)));
      return sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
    }
    return x3max * sqrt(s3);
  }

  // Dogleg step (dogleg.cc) with diag = 1: Gauss-Newton direction if it fits
  // in the trust region, else the scaled-gradient / Gauss-Newton combination.
  __device__ static __forceinline__ void dogleg(const double* r, const double* qtb, double delta,
                                                double* x, double* wa1, double* wa2) {
    const double epsmch = DBL_EPSILON;
#pragma unroll (UNR)
    for (int k = 0; k < N; ++k) {
      const int j = N - 1 - k;
      double sum = 0.;
#pragma unroll (UNR)
      for (int i = j + 1; i < N; ++i) sum += r[rpos(j, i)] * x[i];
      double temp = r[rpos(j, j)];
      if (temp == 0.) {
#pragma unroll (UNR)
        for (int i = 0; i <= j; ++i) {
          double d2 = fabs(r[rpos(i, j)]);
          temp = (temp >= d2) ? temp : d2;
        }
        temp = epsmch * temp;
        if (temp == 0.) temp = epsmch;
      }
      x[j] = (qtb[j] - sum) / temp;
    }
#pragma unroll (UNR)
    for (int j = 0; j < N; ++j) {
      wa1[j] = 0.;
      wa2[j] = x[j];
    }
    double qnorm = hy_enorm<N>(wa2);
    if (qnorm <= delta) return;

#pragma unroll (UNR)
    for (int j = 0; j < N; ++j) {
      double temp = qtb[j];
#pragma unroll (UNR)
      for (int i = j; i < N; ++i) wa1[i] += r[rpos(j, i)] * temp;
    }
    double gnorm = hy_enorm<N>(wa1);
    double sgnorm = 0.;
    double alpha = delta / qnorm;
    if (gnorm != 0.) {
#pragma unroll (UNR)
      for (int j = 0; j < N; ++j) wa1[j] = wa1[j] / gnorm;
#pragma unroll (UNR)
      for (int j = 0; j < N; ++j) {
        double sum = 0.;
#pragma unroll (UNR)
        for (int i = j; i < N; ++i) sum += r[rpos(j, i)] * wa1[i];
        wa2[j] = sum;
      }
      double temp = hy_enorm<N>(wa2);
      sgnorm = gnorm / temp / temp;
      alpha = 0.;
      if (sgnorm < delta) {
        double bnorm = hy_enorm<N>(qtb);
        temp = bnorm / gnorm * (bnorm / qnorm) * (sgnorm / delta);
        double d1 = sgnorm / delta;
        double d2 = temp - delta / qnorm;
        double d3 = delta / qnorm;
        double d4 = sgnorm / delta;
        temp = temp - delta / qnorm * (d1 * d1) + sqrt(d2 * d2 + (1. - d3 * d3) * (1. - d4 * d4));
        d1 = sgnorm / delta;
        alpha = delta / qnorm * (1. - d1 * d1) / temp;
      }
    }
    double mn = (sgnorm <= delta) ? sgnorm : delta;
    double temp = (1. - alpha) * mn;
#pragma unroll (UNR)
    for (int j = 0; j < N; ++j) x[j] = temp * wa1[j] + alpha * x[j];
  }

  // Rank-one update R <- R + u v^T kept upper triangular by Givens rotations
  // (r1updt.cc with m = n).  On exit v and w hold the rotation taus.
  __device__ static __forceinline__ void r1updt(double* s, const double* u, double* v,
                                                double* w) {
    w[N - 1] = s[rpos(N - 1, N - 1)];
#pragma unroll (UNR)
    for (int nmj = 1; nmj < N; ++nmj) {
      const int j = N - 1 - nmj;
      w[j] = 0.;
      if (v[j] != 0.) {
        double c, sn, tau;
        givens(v[j], v[N - 1], fabs(v[N - 1]) < fabs(v[j]), c, sn, tau);
        v[N - 1] = sn * v[j] + c * v[N - 1];
        v[j] = tau;
#pragma unroll (UNR)
        for (int i = j; i < N; ++i) {
          double t = c * s[rpos(j, i)] - sn * w[i];
          w[i] = sn * s[rpos(j, i)] + c * w[i];
          s[rpos(j, i)] = t;
        }
      }
    }
#pragma unroll (UNR)
    for (int i = 0; i < N; ++i) w[i] += v[N - 1] * u[i];
#pragma unroll (UNR)
    for (int j = 0; j < N - 1; ++j) {
      if (w[j] != 0.) {
        double c, sn, tau;
        givens(w[j], s[rpos(j, j)], fabs(s[rpos(j, j)]) < fabs(w[j]), c, sn, tau);
#pragma unroll (UNR)
        for (int i = j; i < N; ++i) {
          double t = c * s[rpos(j, i)] + sn * w[i];
          w[i] = -sn * s[rpos(j, i)] + c * w[i];
          s[rpos(j, i)] = t;
        }
        w[j] = tau;
      }
    }
    s[rpos(N - 1, N - 1)] = w[N - 1];
  }

  // Applies the two rotation sets of r1updt to the columns of Q (r1mpyq.cc).
  __device__ static __forceinline__ void r1mpyq_cols(double* a, const double* v, const double* w) {
#pragma unroll (UNR)
    for (int nmj = 1; nmj < N; ++nmj) {
      const int j = N - 1 - nmj;
      double c, s;
      unpack(v[j], c, s);
#pragma unroll (UNR)
      for (int i = 0; i < N; ++i) {
        double t = c * a[i + N * j] - s * a[i + N * (N - 1)];
        a[i + N * (N - 1)] = s * a[i + N * j] + c * a[i + N * (N - 1)];
        a[i + N * j] = t;
      }
    }
#pragma unroll (UNR)
    for (int j = 0; j < N - 1; ++j) {
      double c, s;
      unpack(w[j], c, s);
#pragma unroll (UNR)
      for (int i = 0; i < N; ++i) {
        double t = c * a[i + N * j] + s * a[i + N * (N - 1)];
        a[i + N * (N - 1)] = -s * a[i + N * j] + c * a[i + N * (N - 1)];
        a[i + N * j] = t;
      }
    }
  }

  // Same rotations applied to the row vector qtf (r1mpyq with m = 1).
  __device__ static __forceinline__ void r1mpyq_row(double* a, const double* v, const double* w) {
#pragma unroll (UNR)
    for (int nmj = 1; nmj < N; ++nmj) {
      const int j = N - 1 - nmj;
      double c, s;
      unpack(v[j], c, s);
      double t = c * a[j] - s * a[N - 1];
      a[N - 1] = s * a[j] + c * a[N - 1];
      a[j] = t;
    }
#pragma unroll (UNR)
    for (int j = 0; j < N - 1; ++j) {
      double c, s;
      unpack(w[j], c, s);
      double t = c * a[j] + s * a[N - 1];
      a[N - 1] = -s * a[j] + c * a[N - 1];
      a[j] = t;
    }
  }
};

}  // namespace mth
