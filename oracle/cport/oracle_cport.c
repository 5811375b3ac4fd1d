/*
 * CPU restatement of the reference's FSAI-preconditioned BiCGSTAB in FP64 C
 * with OpenMP -- TEST INFRASTRUCTURE ONLY: the CPU baseline that bench.py
 * times beside the GPU path (and never part of the product).
 *
 *   fsai factor   : FSAIP_CUDA.cu:92-160 (S = A[P_i,P_i], y = S^-1 e_m, g = y / sqrt(y_m))
 *   BiCGSTAB      : DOGPUP/dMesh.m:1247-1348 (bilinear dots, alph = (v.r0^)/rho0,
 *                   omega in the G-weighted bilinear form, x0 = 0)
 *
 * The reference's own solve is GPU-only (mex kernels driven by MATLAB); it has
 * no CPU solver.  Parallelism: the FSAI rows and the right-hand sides are
 * independent, so both loops run over OpenMP threads; each right-hand side is
 * iterated to its own tolerance.
 *
 * Complex values are interleaved (re, im) doubles.  Matrices are 0-based CSR.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

static inline cplx cmk(double r, double i) { cplx c = {r, i}; return c; }
static inline cplx cmul(cplx a, cplx b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cplx cdiv(cplx a, cplx b) {
  double d = b.re * b.re + b.im * b.im;
  return cmk((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
static inline cplx csub(cplx a, cplx b) { return cmk(a.re - b.re, a.im - b.im); }
static cplx csqrt_principal(cplx z) {
  double m = sqrt(z.re * z.re + z.im * z.im);
  double re = sqrt((m + z.re) / 2), im;
  if (z.im == 0) {
    if (z.re < 0) { re = 0; im = sqrt(-z.re); } else im = 0;
  } else {
    im = (z.im > 0 ? 1.0 : -1.0) * sqrt((m - z.re) / 2);
  }
  return cmk(re, im);
}

int oc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* G values of A = Are + i*Aim (tril CSR rowptr/col) on the pattern (rg, cg). */
int oc_fsai_factor(int n, const int *rowptr, const int *col, const double *Are, const double *Aim, const int *rg,
                   const int *cg, double *Gout) {
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : bad)
  for (int i = 0; i < n; ++i) {
    int gb = rg[i], m = rg[i + 1] - gb;
    if (m < 1 || m > 64) { bad |= 1; continue; }
    cplx S[64][64], y[64];
    for (int a = 0; a < m; ++a) {
      for (int c = 0; c <= a; ++c) {
        int ra = cg[gb + a], cc = cg[gb + c];
        cplx v = cmk(0, 0);
        for (int p = rowptr[ra]; p < rowptr[ra + 1]; ++p)
          if (col[p] == cc) { v = cmk(Are[p], Aim[p]); break; }
        S[a][c] = v;
        S[c][a] = v;
      }
      y[a] = cmk(a == m - 1 ? 1.0 : 0.0, 0.0);
    }
    for (int c = 0; c < m; ++c) { /* elimination with partial pivoting */
      int piv = c;
      double best = S[c][c].re * S[c][c].re + S[c][c].im * S[c][c].im;
      for (int r = c + 1; r < m; ++r) {
        double v = S[r][c].re * S[r][c].re + S[r][c].im * S[r][c].im;
        if (v > best) { best = v; piv = r; }
      }
      if (piv != c) {
        for (int q = c; q < m; ++q) { cplx t = S[c][q]; S[c][q] = S[piv][q]; S[piv][q] = t; }
        cplx t = y[c]; y[c] = y[piv]; y[piv] = t;
      }
      for (int r = c + 1; r < m; ++r) {
        cplx f = cdiv(S[r][c], S[c][c]);
        for (int q = c; q < m; ++q) S[r][q] = csub(S[r][q], cmul(f, S[c][q]));
        y[r] = csub(y[r], cmul(f, y[c]));
      }
    }
    for (int r = m - 1; r >= 0; --r) {
      cplx acc = y[r];
      for (int q = r + 1; q < m; ++q) acc = csub(acc, cmul(S[r][q], y[q]));
      y[r] = cdiv(acc, S[r][r]);
    }
    cplx sq = csqrt_principal(y[m - 1]);
    for (int r = 0; r < m; ++r) {
      cplx g = cdiv(y[r], sq);
      Gout[2 * (gb + r)] = g.re;
      Gout[2 * (gb + r) + 1] = g.im;
    }
  }
  return bad;
}

/* y = (K + i w M) x */
static void spmv_A(int n, const int *rp, const int *cl, const double *K, const double *M, double w, const cplx *x,
                   cplx *y) {
  for (int i = 0; i < n; ++i) {
    double re = 0, im = 0;
    for (int p = rp[i]; p < rp[i + 1]; ++p) {
      cplx v = x[cl[p]];
      double a = K[p], b = w * M[p];
      re += a * v.re - b * v.im;
      im += a * v.im + b * v.re;
    }
    y[i] = cmk(re, im);
  }
}

/* y = G x (complex CSR values) */
static void spmv_G(int n, const int *rp, const int *cl, const cplx *G, const cplx *x, cplx *y) {
  for (int i = 0; i < n; ++i) {
    double re = 0, im = 0;
    for (int p = rp[i]; p < rp[i + 1]; ++p) {
      cplx g = G[p], v = x[cl[p]];
      re += g.re * v.re - g.im * v.im;
      im += g.re * v.im + g.im * v.re;
    }
    y[i] = cmk(re, im);
  }
}

static cplx bil(int n, const cplx *a, const cplx *b) {
  double re = 0, im = 0;
  for (int i = 0; i < n; ++i) {
    re += a[i].re * b[i].re - a[i].im * b[i].im;
    im += a[i].re * b[i].im + a[i].im * b[i].re;
  }
  return cmk(re, im);
}

static double nrm(int n, const cplx *a) {
  double s = 0;
  for (int i = 0; i < n; ++i) s += a[i].re * a[i].re + a[i].im * a[i].im;
  return sqrt(s);
}

/* Solves (K + i w M) X[:,c] = B[:,c] for ncol columns (each [n] complex, column-major)
 * with the reference iteration; per-column iteration counts in iters (may be NULL). */
int oc_bicgstab(int n, const int *rp, const int *cl, const double *K, const double *M, double w, const int *rg,
                const int *cg, const double *G, const int *rt, const int *ct, const double *GT, int ncol,
                const double *B, double *X, double tol, int maxit, int *iters) {
  const cplx *Gc = (const cplx *)G, *GTc = (const cplx *)GT;
#pragma omp parallel
  {
    cplx *r = malloc(sizeof(cplx) * n * 10);
    cplx *rh = r + n, *p = r + 2 * n, *h = r + 3 * n, *v = r + 4 * n, *s = r + 5 * n, *gs = r + 6 * n,
         *z = r + 7 * n, *t = r + 8 * n, *tmp = r + 9 * n;
#pragma omp for schedule(dynamic, 1)
    for (int c = 0; c < ncol; ++c) {
      const cplx *b = (const cplx *)B + (size_t)c * n;
      cplx *x = (cplx *)X + (size_t)c * n;
      memset(x, 0, sizeof(cplx) * n);
      memcpy(r, b, sizeof(cplx) * n);                 /* r = Q - A*0 (dMesh.m:1284-1285) */
      double err0 = nrm(n, r);
      memcpy(rh, r, sizeof(cplx) * n);
      memcpy(p, r, sizeof(cplx) * n);
      cplx rho0 = bil(n, rh, r);
      int it = 0;
      if (err0 > 0) {
        for (it = 1; it <= maxit; ++it) {
          spmv_G(n, rg, cg, Gc, p, tmp);                /* h = G^T G p (:1295-1296) */
          spmv_G(n, rt, ct, GTc, tmp, h);
          spmv_A(n, rp, cl, K, M, w, h, v);             /* :1301 */
          cplx alph = cdiv(bil(n, v, rh), rho0);        /* :1304 */
          for (int i = 0; i < n; ++i) {
            cplx hh = cdiv(h[i], alph), vv = cdiv(v[i], alph);
            h[i] = cmk(x[i].re + hh.re, x[i].im + hh.im);   /* :1305 */
            s[i] = cmk(r[i].re - vv.re, r[i].im - vv.im);   /* :1306 */
          }
          if (nrm(n, s) / err0 < tol) { memcpy(x, h, sizeof(cplx) * n); break; }
          spmv_G(n, rg, cg, Gc, s, gs);                 /* :1315-1322 */
          spmv_G(n, rt, ct, GTc, gs, z);
          spmv_A(n, rp, cl, K, M, w, z, t);
          spmv_G(n, rg, cg, Gc, t, tmp);
          cplx om = cdiv(bil(n, tmp, gs), bil(n, tmp, tmp));   /* :1325 */
          for (int i = 0; i < n; ++i) {
            cplx oz = cmul(om, z[i]), ot = cmul(om, t[i]), ov = cmul(om, v[i]);
            x[i] = cmk(h[i].re + oz.re, h[i].im + oz.im);   /* :1327 */
            r[i] = cmk(s[i].re - ot.re, s[i].im - ot.im);   /* :1328 */
            p[i] = cmk(p[i].re - ov.re, p[i].im - ov.im);   /* :1329 */
          }
          if (nrm(n, r) / err0 < tol) break;            /* :1330-1335 */
          cplx rho = bil(n, rh, r);                      /* :1337-1340 */
          cplx beta = cmul(cdiv(rho, rho0), cdiv(cmk(1, 0), cmul(alph, om)));
          rho0 = rho;
          for (int i = 0; i < n; ++i) {
            cplx bp = cmul(beta, p[i]);
            p[i] = cmk(r[i].re + bp.re, r[i].im + bp.im);
          }
        }
      }
      if (iters) iters[c] = it;
    }
    free(r);
  }
  return 0;
}
