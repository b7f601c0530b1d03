// Device continued fractions and terminators: cf_species (src/asr_chain.f90:67-167), sqrt_tail / cf_green
// (src/reference/asr_greens.f90:12-22, :80-90) and the real Beer-Pettifor asymptote (src/reference/asr_terminator.f90:39-67).
//
// LAPACK zgeev (the reference's eigenvalues of the m x m chain matrix) is replaced by the implicit-shift QL iteration for a
// complex symmetric tridiagonal matrix (eigenvalues only): the EISPACK tql1 / Numerical Recipes tqli scheme carried over
// to complex symmetric matrices with complex plane rotations (Cullum & Willoughby, Lanczos Algorithms for Large Symmetric
// Eigenvalue Computations, Vol. 1, ch. 6, CMTQL1).  dsterf (real tridiagonal eigenvalues) is replaced by Sturm-sequence
// bisection for the extreme eigenvalue.
#pragma once
#include <cfloat>

#include "common.cuh"

namespace asrb {

constexpr int CF_NMAX = 128;   // longest chain the device fractions take

// eigenvalues of the complex symmetric tridiagonal (d[0..n-1], e[0..n-2]) in place in d; e is destroyed.  0 = converged.
__host__ __device__ inline int cs_tridiag_eig(int n, double2* d, double2* e) {
  if (n <= 0) return 0;
  e[n - 1] = make_double2(0.0, 0.0);
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m;
      for (m = l; m < n - 1; ++m) {
        double dd = cmag(d[m]) + cmag(d[m + 1]);
        if (cmag(e[m]) <= DBL_EPSILON * dd || cmag(e[m]) == 0.0) break;
      }
      if (m == l) break;
      if (++iter > 60) return 1;
      double2 g = cdiv(csub(d[l + 1], d[l]), cscale(e[l], 2.0));
      double2 r = csqrt_p(cadd(cmul(g, g), make_double2(1.0, 0.0)));
      double2 gp = cadd(g, r), gm = csub(g, r);
      double2 den = cmag(gp) >= cmag(gm) ? gp : gm;
      g = cadd(csub(d[m], d[l]), cdiv(e[l], den));
      double2 s = make_double2(1.0, 0.0), c = make_double2(1.0, 0.0), p = make_double2(0.0, 0.0);
      bool early = false;
      for (int i = m - 1; i >= l; --i) {
        double2 f = cmul(s, e[i]), b = cmul(c, e[i]);
        r = csqrt_p(cadd(cmul(f, f), cmul(g, g)));
        e[i + 1] = r;
        if (cmag(r) == 0.0) {
          d[i + 1] = csub(d[i + 1], p);
          e[m] = make_double2(0.0, 0.0);
          early = true;
          break;
        }
        s = cdiv(f, r);
        c = cdiv(g, r);
        g = csub(d[i + 1], p);
        r = cadd(cmul(csub(d[i], g), s), cscale(cmul(c, b), 2.0));
        p = cmul(s, r);
        d[i + 1] = cadd(g, p);
        g = csub(cmul(c, r), b);
      }
      if (early) continue;
      d[l] = csub(d[l], p);
      e[l] = g;
      e[m] = make_double2(0.0, 0.0);
    }
  }
  return 0;
}

// extreme (by real part) eigenvalues of the chain matrix with a[m-1] replaced by am; returns 0 on success
__host__ __device__ inline int chain_extremes(const double2* a, const double2* b, int m, double2 am, double2* wd, double2* we,
                                              double2& lo, double2& hi) {
  for (int j = 0; j < m; ++j) wd[j] = a[j];
  wd[m - 1] = am;
  for (int j = 0; j < m - 1; ++j) we[j] = b[j];
  if (cs_tridiag_eig(m, wd, we)) return 1;
  int ilo = 0, ihi = 0;
  for (int j = 1; j < m; ++j) {
    if (wd[j].x < wd[ilo].x) ilo = j;
    if (wd[j].x > wd[ihi].x) ihi = j;
  }
  lo = wd[ilo];
  hi = wd[ihi];
  return 0;
}

// tail parameters (aa, bb) of cf_species (src/asr_chain.f90:80-101): hull extremes, Beer-Pettifor fixed point, avg2 or
// none.  wd, we: work (m).
__host__ __device__ inline void cf_tail_dev(const double2* a, const double2* b, int m, int tail, double2* wd, double2* we,
                                            int* nfall, double2& aa, double2& bb) {
  bool ok = false;
  double2 lo, hi;
  if (m >= 2 && tail != 0) ok = chain_extremes(a, b, m, a[m - 1], wd, we, lo, hi) == 0;
  if (ok) {
    aa = cscale(cadd(lo, hi), 0.5);
    bb = cscale(csub(hi, lo), 0.25);
    if (tail == 2) {   // bp_fixed_point, src/asr_chain.f90:126-156
      bool done = false;
      for (int it = 0; it < 200 && !done; ++it) {
        double2 l1, h1, l2, h2;
        if (chain_extremes(a, b, m, cadd(a[m - 1], bb), wd, we, l1, h1)) { if (nfall) ++*nfall; done = true; break; }
        if (chain_extremes(a, b, m, csub(a[m - 1], bb), wd, we, l2, h2)) { if (nfall) ++*nfall; done = true; break; }
        double2 an = cscale(cadd(h1, l2), 0.5), bn = cscale(csub(h1, l2), 0.25);
        if (cmag(csub(an, aa)) + cmag(csub(bn, bb)) < 1.0e-12 * (1.0 + cmag(bn))) { aa = an; bb = bn; done = true; break; }
        aa = an;
        bb = bn;
      }
      if (!done) {
        if (nfall) ++*nfall;
        chain_extremes(a, b, m, a[m - 1], wd, we, lo, hi);
        aa = cscale(cadd(lo, hi), 0.5);
        bb = cscale(csub(hi, lo), 0.25);
      }
    }
  } else {
    aa = a[m - 1];
    bb = m > 1 ? b[m - 2] : make_double2(0.0, 0.0);
  }
  if (tail == 3 && m >= 3) {
    aa = cscale(cadd(a[m - 1], a[m - 2]), 0.5);
    bb = csqrt_p(cscale(cadd(cmul(b[m - 2], b[m - 2]), cmul(b[m - 3], b[m - 3])), 0.5));
  }
  if (tail == 0) { aa = make_double2(0.0, 0.0); bb = make_double2(0.0, 0.0); }
}

// the square-root terminator of the tail (aa, bb) at z, on the branch with |bb g| minimal (src/asr_chain.f90:103-110)
__host__ __device__ inline double2 cf_tail_term(double2 z, double2 aa, double2 bb) {
  double2 d = csub(z, aa), tl = make_double2(0.0, 0.0);
  if (cmag(bb) >= 1.0e-14) {   // |bb| < 1e-14: no tail
    double2 bb2 = cmul(bb, bb);
    double2 s = csqrt_p(csub(cmul(d, d), cscale(bb2, 4.0)));
    double2 g1 = cdiv(csub(d, s), cscale(bb2, 2.0)), g2 = cdiv(cadd(d, s), cscale(bb2, 2.0));
    tl = cmag(cmul(bb, g1)) <= cmag(cmul(bb, g2)) ? cmul(bb2, g1) : cmul(bb2, g2);
  }
  return tl;
}

// cf_species: g11 of the chain (a, b) of depth m at z with the tail (0 none, 1 hull, 2 bp, 3 avg2).  wd, we: work (m).
__host__ __device__ inline double2 cf_species_dev(const double2* a, const double2* b, int m, double2 z, int tail, double2* wd,
                                                  double2* we, int* nfall, double2* edges) {
  double2 aa, bb;
  cf_tail_dev(a, b, m, tail, wd, we, nfall, aa, bb);
  if (edges) { edges[0] = aa; edges[1] = bb; }
  double2 tl = cf_tail_term(z, aa, bb);
  double2 one = make_double2(1.0, 0.0);
  double2 gt = cdiv(one, csub(csub(z, a[m - 1]), tl));
  for (int j = m - 2; j >= 0; --j) gt = cdiv(one, csub(csub(z, a[j]), cmul(cmul(b[j], b[j]), gt)));
  return gt;
}

// cf_species with the projection f = sum_k c_k prod_{j<k} (b_j gt_{j+1}) gt_1 (src/asr_chain.f90:111-122); closed: the exact
// fraction without tail (cf_closed, src/asr_ed3.f90:221-236).  gt: work (m); wd, we: work (m).
__host__ __device__ inline double2 cf_species_f_dev(const double2* a, const double2* b, const double2* c, int m, double2 z, int tail,
                                                    bool closed, double2* gt, double2* wd, double2* we, int* nfall, double2& f) {
  double2 tl = make_double2(0.0, 0.0);
  if (!closed) {
    double2 aa, bb;
    cf_tail_dev(a, b, m, tail, wd, we, nfall, aa, bb);
    tl = cf_tail_term(z, aa, bb);
  }
  double2 one = make_double2(1.0, 0.0);
  gt[m - 1] = cdiv(one, csub(csub(z, a[m - 1]), tl));
  for (int j = m - 2; j >= 0; --j) gt[j] = cdiv(one, csub(csub(z, a[j]), cmul(cmul(b[j], b[j]), gt[j + 1])));
  f = make_double2(0.0, 0.0);
  double2 prod = gt[0];
  for (int k = 0; k < m; ++k) {
    f = cadd(f, cmul(c[k], prod));
    if (k < m - 1) prod = cmul(prod, cmul(b[k], gt[k + 1]));
  }
  return gt[0];
}

// cf_species with the factors pv_k = [g]_{k1} = gt_1 prod_{j<k} (b_j gt_{j+1}) of the projections f = sum_k c_k pv_k
// (src/asr_chain.f90:111-122, the pv output used by edc_green_proj); pv (m) receives them, the return value is g11.
__host__ __device__ inline double2 cf_species_pv_dev(const double2* a, const double2* b, int m, double2 z, int tail, double2* pv,
                                                     double2* wd, double2* we, int* nfall) {
  double2 aa, bb;
  cf_tail_dev(a, b, m, tail, wd, we, nfall, aa, bb);
  double2 tl = cf_tail_term(z, aa, bb);
  double2 one = make_double2(1.0, 0.0);
  pv[m - 1] = cdiv(one, csub(csub(z, a[m - 1]), tl));   // gt in place, then turned into the products
  for (int j = m - 2; j >= 0; --j) pv[j] = cdiv(one, csub(csub(z, a[j]), cmul(cmul(b[j], b[j]), pv[j + 1])));
  double2 g11 = pv[0], prod = pv[0];
  for (int k = 0; k < m; ++k) {
    double2 gnext = k < m - 1 ? pv[k + 1] : make_double2(0.0, 0.0);
    pv[k] = prod;
    if (k < m - 1) prod = cmul(prod, cmul(b[k], gnext));
  }
  return g11;
}

// ---- real chains (plain mode)
__host__ __device__ inline int sturm_count(int n, const double* d, const double* e, double x) {
  int cnt = 0;
  double q = d[0] - x;
  if (q < 0) ++cnt;
  for (int i = 1; i < n; ++i) {
    if (q == 0.0) q = DBL_EPSILON * (fabs(e[i - 1]) + DBL_MIN);
    q = d[i] - x - e[i - 1] * e[i - 1] / q;
    if (q < 0) ++cnt;
  }
  return cnt;
}
__host__ __device__ inline double tridiag_extreme(int n, const double* d, const double* e, bool upper) {
  double lo = d[0], hi = d[0];
  for (int i = 0; i < n; ++i) {
    double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
  }
  double span = hi - lo;
  lo -= 1e-12 * (span + 1.0);
  hi += 1e-12 * (span + 1.0);
  int target = upper ? n : 1;
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_count(n, d, e, mid) >= target) hi = mid; else lo = mid;
  }
  return 0.5 * (lo + hi);
}
// bp_asymptote (src/reference/asr_terminator.f90:39-67); wd: work (n)
__host__ __device__ inline void bp_asymptote_dev(const double* a, const double* b, int n, double* wd, double& ainf, double& binf) {
  double A = 0.5 * (a[n - 1] + a[n - 2]);
  double B = sqrt(0.5 * (b[n - 1] * b[n - 1] + b[n - 2] * b[n - 2]));
  for (int it = 0; it < 500; ++it) {
    for (int i = 0; i < n; ++i) wd[i] = a[i];
    wd[n - 1] = a[n - 1] + B;
    double ep = tridiag_extreme(n, wd, b, true);
    wd[n - 1] = a[n - 1] - B;
    double em = tridiag_extreme(n, wd, b, false);
    double an = 0.5 * (ep + em), bn = 0.25 * (ep - em);
    bool conv = fabs(an - A) + fabs(bn - B) < 1.0e-13;
    A = an;
    B = bn;
    if (conv) break;
  }
  ainf = A;
  binf = B;
}
// sqrt_tail + cf_green (src/reference/asr_greens.f90:12-22, :80-90)
__host__ __device__ inline double2 terminated_green_dev(const double* a, const double* b, int n, double2 z, double ainf, double binf,
                                                        bool has_tail) {
  double2 tl = make_double2(0.0, 0.0);
  if (has_tail) {
    double2 w = make_double2(z.x - ainf, z.y);
    double2 s = csqrt_p(csub(cmul(w, w), make_double2(4.0 * binf * binf, 0.0)));
    double d2 = 2.0 * binf * binf;
    double2 g1 = cscale(csub(w, s), 1.0 / d2), g2 = cscale(cadd(w, s), 1.0 / d2);
    double2 g = cmag(g1) <= cmag(g2) ? g1 : g2;
    tl = cscale(g, binf * binf);
  }
  double2 one = make_double2(1.0, 0.0);
  double2 g = cdiv(one, csub(make_double2(z.x - a[n - 1], z.y), tl));
  for (int i = n - 2; i >= 0; --i) g = cdiv(one, csub(make_double2(z.x - a[i], z.y), cscale(g, b[i] * b[i])));
  return g;
}


// ---- reverse mode of cf_species (tails none, hull, avg2): abar_k += w dG/da_k, bbar_k += w dG/db_k.  G is holomorphic in
// (a, b) away from the branch choices, so the complex derivatives compose.  The hull edges are extreme eigenvalues of
// the chain matrix T; for a simple eigenvalue of a complex symmetric matrix d(lambda) = v^T dT v / (v^T v), with v from
// inverse iteration on T - lambda.  wd, we, wx: work (m).  Returns 0 on success.
__host__ __device__ inline int tridiag_solve_shift(int m, const double2* a, const double2* b, double2 lam, const double2* rhs,
                                                   double2* x, double2* wd, double2* we) {
  // (T - lam) x = rhs, Thomas algorithm on the complex symmetric tridiagonal (no pivoting; lam is perturbed off the
  // eigenvalue by the caller)
  double2 dd = csub(a[0], lam);
  if (cmag(dd) == 0.0) dd = make_double2(1e-300, 0.0);
  wd[0] = dd;
  x[0] = rhs[0];
  for (int j = 1; j < m; ++j) {
    double2 l = cdiv(b[j - 1], wd[j - 1]);
    we[j - 1] = l;
    double2 d = csub(csub(a[j], lam), cmul(l, b[j - 1]));
    if (cmag(d) == 0.0) d = make_double2(1e-300, 0.0);
    wd[j] = d;
    x[j] = csub(rhs[j], cmul(l, x[j - 1]));
  }
  x[m - 1] = cdiv(x[m - 1], wd[m - 1]);
  for (int j = m - 2; j >= 0; --j) x[j] = cdiv(csub(x[j], cmul(b[j], x[j + 1])), wd[j]);
  return 0;
}

// eigenvector t (scaled to max modulus 1) of the complex symmetric tridiagonal (a, b) at the simple eigenvalue lam: two
// steps of inverse iteration at a shift next to lam; returns t.t (the bilinear, not the Hermitian, square)
__host__ __device__ inline double2 eig_vec(int m, const double2* a, const double2* b, double2 lam, double2* v, double2* t,
                                           double2* wd, double2* we) {
  double sc = 0.0;
  for (int j = 0; j < m; ++j) sc = fmax(sc, cmag(a[j]) + (j < m - 1 ? cmag(b[j]) : 0.0));
  double2 mu = cadd(lam, make_double2(1e-10 * (sc + 1.0), 1e-10 * (sc + 1.0)));
  for (int j = 0; j < m; ++j) t[j] = make_double2(1.0 / sqrt((double)m), 0.0);
  for (int it = 0; it < 3; ++it) {
    tridiag_solve_shift(m, a, b, mu, t, v, wd, we);
    double nr = 0.0;
    for (int j = 0; j < m; ++j) nr = fmax(nr, cmag(v[j]));
    for (int j = 0; j < m; ++j) t[j] = cscale(v[j], 1.0 / nr);
  }
  double2 vv = make_double2(0.0, 0.0);
  for (int j = 0; j < m; ++j) vv = cadd(vv, cmul(t[j], t[j]));
  return vv;
}

// abar_j += w dlam/da_j, bbar_j += w dlam/db_j with dlam = v^T dT v / (v^T v)
__host__ __device__ inline void eig_grad(int m, const double2* a, const double2* b, double2 lam, double2 w, double2* abar,
                                         double2* bbar, double2* v, double2* t, double2* wd, double2* we) {
  double2 vv = eig_vec(m, a, b, lam, v, t, wd, we);
  double2 f = cdiv(w, vv);
  for (int j = 0; j < m; ++j) abar[j] = cadd(abar[j], cmul(f, cmul(t[j], t[j])));
  for (int j = 0; j < m - 1; ++j) bbar[j] = cadd(bbar[j], cmul(f, cscale(cmul(t[j], t[j + 1]), 2.0)));
}

// dlam / da_{m-1} = v_{m-1}^2 / (v^T v): the sensitivity of the eigenvalue to the last diagonal entry
__host__ __device__ inline double2 eig_last_sens(int m, const double2* a, const double2* b, double2 lam, double2* v, double2* t,
                                                 double2* wd, double2* we) {
  double2 vv = eig_vec(m, a, b, lam, v, t, wd, we);
  return cdiv(cmul(t[m - 1], t[m - 1]), vv);
}

// w: seed; work arrays of length >= m each: gt, v, t, wd, we.  Returns G.
__host__ __device__ inline double2 cf_species_adjoint(const double2* a, const double2* b, int m, double2 z, int tail, double2 w,
                                                       double2* abar, double2* bbar, double2* gt, double2* v, double2* t, double2* wd,
                                                       double2* we) {
  // forward: tail parameters
  double2 aa = make_double2(0, 0), bb = make_double2(0, 0), lo, hi, ep = make_double2(0, 0), em = make_double2(0, 0);
  int kind = 0;   // 0 none / finite, 1 hull, 2 last coefficients, 3 avg2, 4 Beer-Pettifor fixed point, 5 tail held fixed
  if (tail == 2 && m >= 2 && chain_extremes(a, b, m, a[m - 1], wd, we, lo, hi) == 0) {
    // the fixed point as cf_tail_dev iterates it (src/asr_chain.f90:126-156): converged -> differentiated implicitly;
    // not converged -> the hull values (differentiated as the hull); an eigenvalue failure keeps the last iterate, whose
    // dependence on (a, b) is not followed (kind 5)
    aa = cscale(cadd(lo, hi), 0.5);
    bb = cscale(csub(hi, lo), 0.25);
    kind = 1;
    for (int it = 0; it < 200; ++it) {
      double2 l1, h1, l2, h2;
      if (chain_extremes(a, b, m, cadd(a[m - 1], bb), wd, we, l1, h1) ||
          chain_extremes(a, b, m, csub(a[m - 1], bb), wd, we, l2, h2)) { kind = 5; break; }
      double2 an = cscale(cadd(h1, l2), 0.5), bn = cscale(csub(h1, l2), 0.25);
      if (cmag(csub(an, aa)) + cmag(csub(bn, bb)) < 1.0e-12 * (1.0 + cmag(bn))) {
        aa = an; bb = bn; ep = h1; em = l2; kind = 4;
        break;
      }
      aa = an;
      bb = bn;
    }
    if (kind == 1) {   // not converged within 200 iterations: the hull
      aa = cscale(cadd(lo, hi), 0.5);
      bb = cscale(csub(hi, lo), 0.25);
    }
  } else if (tail == 3 && m >= 3) {
    aa = cscale(cadd(a[m - 1], a[m - 2]), 0.5);
    bb = csqrt_p(cscale(cadd(cmul(b[m - 2], b[m - 2]), cmul(b[m - 3], b[m - 3])), 0.5));
    kind = 3;
  } else if (tail == 1 && m >= 2 && chain_extremes(a, b, m, a[m - 1], wd, we, lo, hi) == 0) {
    aa = cscale(cadd(lo, hi), 0.5);
    bb = cscale(csub(hi, lo), 0.25);
    kind = 1;
  } else if (tail != 0 && m >= 1) {   // eigenvalue failure or m = 1: the last coefficients (src/asr_chain.f90:95)
    aa = a[m - 1];
    bb = m > 1 ? b[m - 2] : make_double2(0.0, 0.0);
    kind = 2;
  }
  double2 d = csub(z, aa), tl = make_double2(0, 0), sroot = make_double2(0, 0);
  double sig = 0.0;
  bool has_tail = cmag(bb) >= 1.0e-14;
  if (has_tail) {
    double2 bb2 = cmul(bb, bb);
    sroot = csqrt_p(csub(cmul(d, d), cscale(bb2, 4.0)));
    double2 g1 = cdiv(csub(d, sroot), cscale(bb2, 2.0)), g2 = cdiv(cadd(d, sroot), cscale(bb2, 2.0));
    if (cmag(cmul(bb, g1)) <= cmag(cmul(bb, g2))) { tl = cmul(bb2, g1); sig = 1.0; }
    else { tl = cmul(bb2, g2); sig = -1.0; }
  }
  double2 one = make_double2(1.0, 0.0);
  gt[m - 1] = cdiv(one, csub(csub(z, a[m - 1]), tl));
  for (int j = m - 2; j >= 0; --j) gt[j] = cdiv(one, csub(csub(z, a[j]), cmul(cmul(b[j], b[j]), gt[j + 1])));
  const double2 G = gt[0];
  // reverse: gbar_j is the adjoint of gt_j
  double2 gbar = w;
  double2 tbar = make_double2(0, 0);
  for (int j = 0; j < m; ++j) {
    double2 Dbar = cmul(cscale(cmul(gt[j], gt[j]), -1.0), gbar);   // d gt / dD = -gt^2
    abar[j] = csub(abar[j], Dbar);
    if (j < m - 1) {
      bbar[j] = csub(bbar[j], cscale(cmul(cmul(b[j], gt[j + 1]), Dbar), 2.0));
      gbar = csub(make_double2(0, 0), cmul(cmul(b[j], b[j]), Dbar));
    } else {
      tbar = csub(make_double2(0, 0), Dbar);
    }
  }
  if (has_tail && kind != 0) {
    // T = (d - sig s) / 2, s^2 = d^2 - 4 bb^2, d = z - aa
    double2 aabar = cscale(cmul(tbar, csub(cscale(cdiv(d, sroot), sig), one)), 0.5);
    double2 bbbar = cmul(tbar, cscale(cdiv(bb, sroot), 2.0 * sig));
    if (kind == 3) {
      abar[m - 1] = cadd(abar[m - 1], cscale(aabar, 0.5));
      abar[m - 2] = cadd(abar[m - 2], cscale(aabar, 0.5));
      double2 f = cdiv(bbbar, cscale(bb, 2.0));   // d bb / d b_j = b_j / (2 bb)
      bbar[m - 2] = cadd(bbar[m - 2], cmul(f, b[m - 2]));
      bbar[m - 3] = cadd(bbar[m - 3], cmul(f, b[m - 3]));
    } else if (kind == 2) {
      abar[m - 1] = cadd(abar[m - 1], aabar);
      if (m > 1) bbar[m - 2] = cadd(bbar[m - 2], bbbar);
    } else if (kind == 4) {
      // bb = phi(bb) = (ep(a_m + bb) - em(a_m - bb)) / 4 and aa = (ep + em) / 2 at the fixed point.  With the
      // sensitivities pv = d ep / d a_m, pu = d em / d a_m (eigenvectors of the two shifted chain matrices):
      // d phi / d bb = (pv + pu) / 4, partial d aa / d bb = (pv - pu) / 2, and the adjoint of the fixed point
      // lam = (bbbar + aabar (pv - pu) / 2) / (1 - (pv + pu) / 4); the eigenvalue seeds are aabar / 2 +- lam / 4.
      double2* am = gt;   // gt is no longer needed: the shifted diagonal
      for (int j = 0; j < m; ++j) am[j] = a[j];
      am[m - 1] = cadd(a[m - 1], bb);
      double2 pv = eig_last_sens(m, am, b, ep, v, t, wd, we);
      am[m - 1] = csub(a[m - 1], bb);
      double2 pu = eig_last_sens(m, am, b, em, v, t, wd, we);
      double2 den = csub(one, cscale(cadd(pv, pu), 0.25));
      double2 lam = cdiv(cadd(bbbar, cmul(aabar, cscale(csub(pv, pu), 0.5))), den);
      double2 wp = cadd(cscale(aabar, 0.5), cscale(lam, 0.25)), wm = csub(cscale(aabar, 0.5), cscale(lam, 0.25));
      am[m - 1] = cadd(a[m - 1], bb);
      eig_grad(m, am, b, ep, wp, abar, bbar, v, t, wd, we);
      am[m - 1] = csub(a[m - 1], bb);
      eig_grad(m, am, b, em, wm, abar, bbar, v, t, wd, we);
    } else if (kind == 5) {
      // tail held fixed
    } else {
      // aa = (lo + hi)/2, bb = (hi - lo)/4
      double2 wlo = csub(cscale(aabar, 0.5), cscale(bbbar, 0.25)), whi = cadd(cscale(aabar, 0.5), cscale(bbbar, 0.25));
      eig_grad(m, a, b, lo, wlo, abar, bbar, v, t, wd, we);
      eig_grad(m, a, b, hi, whi, abar, bbar, v, t, wd, we);
    }
  }
  return G;
}

// kernels of cf.cu
__global__ void k_cf_eval(const double2* a, const double2* b, const int* m, int ld, int nchain, const double2* z, int nz, int tail,
                          double2* g, double2* edges, int* nfall);
__global__ void k_real_tail(const double* a, const double* b, const int* n, int ld, int nchain, int method, double* ainf,
                            double* binf);
__global__ void k_real_green(const double* a, const double* b, const int* n, int ld, int nchain, const double* ainf,
                             const double* binf, int method, const double2* z, int nz, double2* g);

}  // namespace asrb
