/*
 * bs_oracle.c -- FP64 C restatement of core/BiotSavart.m:36-119 (test
 * infrastructure: the checker and the timed CPU baseline, never the product).
 *
 * For every target (loops k, j, i of BiotSavart.m:80-82) it evaluates every
 * filament with the formulas of :89-109 in MATLAB's operation order, zeroes
 * NaN/Inf terms and terms with r1>co and r2>co (:111), and sums over the
 * filament dimensions in MATLAB's nesting sum(sum(sum(.,1),3),4) (:113-115),
 * each sum sequential. Targets are split across OpenMP threads.
 */
#include <math.h>
#include <stddef.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double k4pi = 4.0 * 3.141592653589793;

/* visc = 0: cut-off core with squared cut-off d; visc = 1: Vatistas index n = d. */
int bs_oracle_eval(const double *F1, const double *F2, const double *gamma, const double *rc,
                   const long long fd[4], const double *P, const long long pd[4], int visc,
                   double d, double co, double *uind, int nthreads) {
  const long long fs = fd[0], ft = fd[2], fb = fd[3];
  const long long ns = pd[0], nt = pd[2], nb = pd[3];
  const long long np = ns * nt * nb;
  const double n = visc ? d : 0.0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
  for (long long t = 0; t < np; ++t) {
    const long long i = t % ns, jk = t / ns;
    const double px = P[i + ns * (0 + 3 * jk)];
    const double py = P[i + ns * (1 + 3 * jk)];
    const double pz = P[i + ns * (2 + 3 * jk)];
    double u3[3] = {0.0, 0.0, 0.0};
    for (long long kb = 0; kb < fb; ++kb) {
      double sk[3] = {0.0, 0.0, 0.0};
      for (long long j = 0; j < ft; ++j) {
        double sj[3] = {0.0, 0.0, 0.0};
        for (long long m = 0; m < fs; ++m) {
          const long long q = m + fs * 3 * (j + ft * kb);
          const long long g = m + fs * (j + ft * kb);
          const double x1 = F1[q], y1 = F1[q + fs], z1 = F1[q + 2 * fs];
          const double x2 = F2[q], y2 = F2[q + fs], z2 = F2[q + 2 * fs];
          const double x2x1 = x2 - x1, y2y1 = y2 - y1, z2z1 = z2 - z1;
          const double L = x2x1 * x2x1 + y2y1 * y2y1 + z2z1 * z2z1;
          const double pxx1 = px - x1, pyy1 = py - y1, pzz1 = pz - z1;
          const double pxx2 = px - x2, pyy2 = py - y2, pzz2 = pz - z2;
          const double r1 = sqrt(pxx1 * pxx1 + pyy1 * pyy1 + pzz1 * pzz1);
          const double r2 = sqrt(pxx2 * pxx2 + pyy2 * pyy2 + pzz2 * pzz2);
          const double r1dr2 = pxx1 * pxx2 + pyy1 * pyy2 + pzz1 * pzz2;
          const double r1tr2 = r1 * r2;
          double ubar;
          if (n != 0.0) {
            const double ld = x2x1 * pxx1 + y2y1 * pyy1 + z2z1 * pzz1;
            double Cnu = r1 * r1 - (ld * ld) / L;
            if (n == 2.0) /* pow(x,2) is exact; x^(-1/2) as 1/sqrt(x), within 1 ulp of pow */
              Cnu = Cnu * (1.0 / sqrt(rc[g] * rc[g] + Cnu * Cnu));
            else
              Cnu = Cnu * pow(pow(rc[g], n) + pow(Cnu, n), -1.0 / n);
            ubar = Cnu * gamma[g] / k4pi * (r1 + r2) / (r1tr2 * (r1tr2 + r1dr2));
          } else {
            ubar = (gamma[g] / k4pi) * (r1 + r2) / (r1tr2 * (r1tr2 + r1dr2) + (d * L));
          }
          if (isnan(ubar) || isinf(ubar) || (r1 > co && r2 > co)) ubar = 0.0;
          sj[0] += ubar * (pyy1 * pzz2 - pzz1 * pyy2);
          sj[1] += ubar * (pzz1 * pxx2 - pxx1 * pzz2);
          sj[2] += ubar * (pxx1 * pyy2 - pyy1 * pxx2);
        }
        sk[0] += sj[0];
        sk[1] += sj[1];
        sk[2] += sj[2];
      }
      u3[0] += sk[0];
      u3[1] += sk[1];
      u3[2] += sk[2];
    }
    uind[i + ns * (0 + 3 * jk)] = u3[0];
    uind[i + ns * (1 + 3 * jk)] = u3[1];
    uind[i + ns * (2 + 3 * jk)] = u3[2];
  }
  return 0;
}

/* Filament lengths, core/FilamentLength.m:27-44. */
void bs_oracle_length(const double *F1, const double *F2, const long long fd[4], double *L) {
  const long long fs = fd[0], n = fd[0] * fd[2] * fd[3];
  for (long long f = 0; f < n; ++f) {
    const long long m = f % fs, jk = f / fs;
    const long long q = m + fs * 3 * jk;
    const double dx = F2[q] - F1[q], dy = F2[q + fs] - F1[q + fs], dz = F2[q + 2 * fs] - F1[q + 2 * fs];
    L[f] = sqrt(dx * dx + dy * dy + dz * dz);
  }
}
