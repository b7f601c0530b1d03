// asr_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A CPU restatement (C++17, FP64) of the recursion hot path of mavensgroup/asr, used ONLY as the checker by tests/,
// by __graft_entry__.smoke() and by bench.py's cpu_baseline / reference legs.  Nothing in asr_b200/ links, imports or
// calls this file.  Every routine cites the reference Fortran it restates (paths relative to the asr project root).
//
// Parity pins: the golden complex chains and known-answer tests of test/test_terminators.f90 (tests/golden/), the
// exact-enumeration toy models of test_slow/test_augcls.f90 (ring; dense numpy solve), the reduced == unreduced
// dense-solve check of test/test_augcls_project.f90, the node counts the reference prints for its shipped examples
// (example/reference/*/asr.out), the task-count invariance of test/test_augcls_threads.f90, and the sc-band contour
// moments of test/test_contour.f90 against exact band integrals.  LAPACK zgeev / dsterf (external, no pinned version; MKL or
// OpenBLAS) are replaced by published algorithms: shifted complex Hessenberg QR (Golub & Van Loan, Alg. 7.5.1 with
// Wilkinson shifts) and Sturm-sequence bisection (Wilkinson 1965); tests check both against scipy's LAPACK.
//
// Conventions: arrays cross the ABI in Fortran (column-major) layout; stored site/node indices are 1-based as in the
// reference; internal loops are 0-based.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;
static const double PI = 3.14159265358979323846264338327950288;

static thread_local std::string g_err;
static int fail(const char* msg) { g_err = msg; return 1; }

extern "C" const char* orc_last_error() { return g_err.c_str(); }

// ===================================================================================================== hashed store
// src/asr_augspace.f90:33-116 (store_t, hash_key, find_or_add, find_state)
struct Store {
  int n = 0;
  std::vector<int> site, start, len, level, orb, data;
  std::vector<int> table;
  int64_t tmask = 0;
  void init(int cap) {
    site.reserve(cap); start.reserve(cap); len.reserve(cap); level.reserve(cap); orb.reserve(cap);
    int64_t tsz = 1024;
    while (tsz < 4 * (int64_t)cap) tsz *= 2;
    table.assign(tsz, 0); tmask = tsz - 1;
  }
  static int64_t hash_key(int s, const int* cfg, int nc) {   // src/asr_augspace.f90:59-69
    uint64_t h = (uint64_t)(1469598103LL + (int64_t)s * 1099511LL);
    for (int i = 0; i < nc; ++i) {
      h ^= (uint64_t)((int64_t)cfg[i] + 1234567LL);
      h = (h * 16777619ULL) & 2147483647ULL;
    }
    return (int64_t)(h & 2147483647ULL);
  }
  bool same(int j, int s, const int* cfg, int nc) const {
    if (site[j - 1] != s || len[j - 1] != nc) return false;
    for (int q = 0; q < nc; ++q) if (data[start[j - 1] + q] != cfg[q]) return false;
    return true;
  }
  int find(int s, const int* cfg, int nc) const {           // find_state :102-116
    int64_t h = hash_key(s, cfg, nc) & tmask;
    for (;;) {
      int j = table[h];
      if (j == 0) return 0;
      if (same(j, s, cfg, nc)) return j;
      h = (h + 1) & tmask;
    }
  }
  void rehash() {
    int64_t tsz = 2 * (tmask + 1);
    table.assign(tsz, 0); tmask = tsz - 1;
    for (int j = 1; j <= n; ++j) {
      int64_t h = hash_key(site[j - 1], &data[start[j - 1]], len[j - 1]) & tmask;
      while (table[h] != 0) h = (h + 1) & tmask;
      table[h] = j;
    }
  }
  int find_or_add(int s, const int* cfg, int nc, int lev, bool& isnew) {   // find_or_add :72-99
    int64_t h = hash_key(s, cfg, nc) & tmask;
    for (;;) {
      int j = table[h];
      if (j == 0) break;
      if (same(j, s, cfg, nc)) { isnew = false; return j; }
      h = (h + 1) & tmask;
    }
    ++n;
    site.push_back(s); len.push_back(nc); level.push_back(lev); orb.push_back(1);
    start.push_back((int)data.size());
    for (int q = 0; q < nc; ++q) data.push_back(cfg[q]);
    table[h] = n;
    isnew = true;
    if (4 * (int64_t)n > tmask) rehash();
    return n;
  }
};

// ===================================================================================================== configurations
// src/asr_augcls.f90:207-235 (get_state, set_state), :494-550 (canon_node, sort_small, uniq3)
static int get_state(const std::vector<int>& cfg, int r, int nsm) {
  for (int c : cfg) if (c / nsm == r) return c % nsm;
  return 0;
}
static std::vector<int> set_state(const std::vector<int>& cfg, int r, int k, int nsm) {
  std::vector<int> t;
  t.reserve(cfg.size() + 1);
  for (int c : cfg) if (c / nsm != r) t.push_back(c);
  if (k > 0) {
    t.push_back(r * nsm + k);
    int i = (int)t.size() - 1;
    while (i > 0) {
      if (t[i - 1] <= t[i]) break;
      std::swap(t[i], t[i - 1]); --i;
    }
  }
  return t;
}
static void sort_small(std::vector<int>& a) {
  for (size_t i = 1; i < a.size(); ++i) {
    int t = a[i]; long j = (long)i - 1;
    while (j >= 0) { if (a[j] <= t) break; a[j + 1] = a[j]; --j; }
    a[j + 1] = t;
  }
}
// perm: Fortran perm(nsite, nop), 1-based values
static void canon_node(const int* perm, int nsite, int nop, int nsm, int s, const std::vector<int>& cfg,
                       int& csite, std::vector<int>& ccfg, int& osize, int& gbest) {
  const int n = (int)cfg.size();
  std::vector<int> c2(n);
  csite = INT32_MAX; ccfg.assign(n, INT32_MAX);
  int ntie = 0; gbest = 1;
  for (int iop = 1; iop <= nop; ++iop) {
    const int* p = perm + (size_t)(iop - 1) * nsite;
    int s2 = p[s - 1];
    for (int k = 0; k < n; ++k) c2[k] = p[cfg[k] / nsm - 1] * nsm + cfg[k] % nsm;
    sort_small(c2);
    bool better = false, equal = false;
    if (s2 < csite) better = true;
    else if (s2 == csite) {
      equal = true;
      for (int k = 0; k < n; ++k) {
        if (c2[k] < ccfg[k]) { better = true; equal = false; break; }
        else if (c2[k] > ccfg[k]) { equal = false; break; }
      }
    }
    if (better) { csite = s2; ccfg = c2; ntie = 1; gbest = iop; }
    else if (equal) ++ntie;
  }
  osize = nop / ntie;
}

// ===================================================================================================== local basis
// src/asr_augcls.f90:73-91 (augn_basis), :190-205 (class_mt)
static void augn_basis(const std::vector<double>& conc, std::vector<double>& phi /* (ns, ns) col-major */) {
  int ns = (int)conc.size();
  phi.assign((size_t)ns * ns, 0.0);
  auto P = [&](int l, int s) -> double& { return phi[l + (size_t)ns * s]; };
  for (int s = 0; s < ns; ++s) P(0, s) = 1.0;
  for (int l = 1; l < ns; ++l) {
    for (int s = 0; s < ns; ++s) P(l, s) = 0.0;
    P(l, l - 1) = 1.0;
    for (int pass = 0; pass < 2; ++pass)
      for (int m = 0; m < l; ++m) {
        double ip = 0.0;
        for (int s = 0; s < ns; ++s) ip += conc[s] * P(m, s) * P(l, s);
        for (int s = 0; s < ns; ++s) P(l, s) = P(l, s) - ip * P(m, s);
      }
    double nrm = 0.0;
    for (int s = 0; s < ns; ++s) nrm += conc[s] * P(l, s) * P(l, s);
    nrm = std::sqrt(nrm);
    for (int s = 0; s < ns; ++s) P(l, s) = P(l, s) / nrm;
  }
}
// mt(l, k, j) for one class (nsm x nsm x nsm, col-major); conc has the nsc species of the class
static void class_mt(const std::vector<double>& conc, int nsm, double* mt) {
  for (int q = 0; q < nsm * nsm * nsm; ++q) mt[q] = 0.0;
  std::vector<int> sup;
  for (int j = 0; j < (int)conc.size(); ++j) if (conc[j] > 0.0) sup.push_back(j);
  int n = (int)sup.size();
  std::vector<double> cs(n);
  for (int j = 0; j < n; ++j) cs[j] = conc[sup[j]];
  std::vector<double> phi;
  augn_basis(cs, phi);
  for (int l = 0; l < n; ++l)
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        mt[l + nsm * (k + nsm * (size_t)sup[j])] = cs[j] * phi[l + (size_t)n * j] * phi[k + (size_t)n * j];
}

// ===================================================================================================== operator
struct Op {
  int nn = 0, nslot = 0, nop = 1, nsmax = 1, ncls = 0, nsp = 0, ntype = 1, nsite = 0, start_l = 1;
  std::vector<int> nsc, spc;      // spc(ldspc, ncls)
  int ldspc = 1;
  std::vector<int> stype;         // (nsite)
  std::vector<double> mt;         // (nsm, nsm, nsm, ncls)
  std::vector<double> c, d, o, e; // (9, nsp)
  std::vector<double> block0;     // (9, 9, ntype)
  std::vector<double> btab;       // (9, 9, ns, nop, ntype)
  std::vector<int> flipr, flipg, hopr, hopg, lst, site, ncl, level, frozen;
  std::vector<double> norb, sq;
  std::vector<int> pi;            // (9, nop)
  std::vector<double> sg, chi, csg, dmat;
  std::vector<int> stab_ptr, stab;
  int spcv(int k, int kap) const { return spc[k + (size_t)ldspc * kap]; }   // 0-based k, kap; 1-based species value
};

// src/asr_augcls.f90:596-823 (build_augcls_operator)
// graph: nbr_ptr(n+1), nbr (1-based); conc(ldspc, ncls); cls(n); perm(n, nop); dmat(9,9,nop); flippable (n) or null;
// stype (n) or null; block(9,9,nsb,ntype) with nsb >= nslot; block0(9,9,ntype) or null.
// tsite (ntarget, 1-based sites) optional: target links tnode(nsm, ntarget) (1-based node, 0 absent), tgop (1-based op)
static int build_impl(int n, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc, int ldspc,
                      const double* conc, int nsp, const int* cls, const int* perm, int nop, const double* dmat,
                      int start, int maxlevel, int maxrank, const int* flippable, const int* stype,
                      const double* block, int nsb, int ntb, const double* block0, const int* tsite, int ntarget, int* tnode,
                      int* tgop, void** handle) {
  *handle = nullptr;
  for (int i = 0; i < n; ++i) if (perm[i] != i + 1) return fail("build_augcls_operator: operation 1 must be the identity");
  for (int g = 0; g < nop; ++g) {
    const int* p = perm + (size_t)g * n;
    if (p[start - 1] != start) return fail("build_augcls_operator: the group does not fix the start site");
    for (int i = 0; i < n; ++i) if (cls[p[i] - 1] != cls[i]) return fail("build_augcls_operator: an operation does not preserve the site classes");
  }
  Op* op = new Op();
  op->nsite = n;
  op->stype.assign(n, 1);
  if (stype) for (int i = 0; i < n; ++i) op->stype[i] = stype[i];
  int nty = *std::max_element(op->stype.begin(), op->stype.end());
  if (*std::min_element(op->stype.begin(), op->stype.end()) < 1 || nty > ntb) { delete op; return fail("build_augcls_operator: site type without a bond table"); }
  op->ntype = nty;
  int nsm = 0;
  for (int k = 0; k < ncls; ++k) nsm = std::max(nsm, nsc[k]);
  int rkmax = maxrank > 0 ? maxrank : INT32_MAX;
  std::vector<char> canflip(n, 1);
  if (flippable) for (int i = 0; i < n; ++i) canflip[i] = flippable[i] != 0;
  std::vector<int> nst(n);
  for (int r = 0; r < n; ++r) nst[r] = canflip[r] ? nsc[cls[r] - 1] : 1;
  Store st; st.init(4096);
  std::vector<int> cfg0, ccf;
  int cs, osz, gb;
  canon_node(perm, n, nop, nsm, start, cfg0, cs, ccf, osz, gb);
  if (osz != 1) { delete op; return fail("build_augcls_operator: start site is not invariant under the group"); }
  bool isnew;
  int idx = st.find_or_add(cs, ccf.data(), (int)ccf.size(), 0, isnew);
  st.orb[idx - 1] = 1;
  // serial breadth-first closure: node order = order of first insertion over (node, k1, k2, f)
  for (int i = 1; i <= st.n; ++i) {
    int lev = st.level[i - 1];
    if (lev >= maxlevel) continue;
    int r = st.site[i - 1];
    std::vector<int> c0(st.data.begin() + st.start[i - 1], st.data.begin() + st.start[i - 1] + st.len[i - 1]);
    int deg_r = nbr_ptr[r] - nbr_ptr[r - 1];
    for (int k1 = 0; k1 <= deg_r; ++k1) {
      int r1 = (k1 == 0) ? r : nbr[nbr_ptr[r - 1] + k1 - 2];
      if (r1 == 0) continue;
      if (r1 < 0) { delete op; return fail("build_augcls_operator: the closure reaches the edge of the site cluster"); }
      int deg_r1 = nbr_ptr[r1] - nbr_ptr[r1 - 1];
      for (int k2 = 0; k2 <= deg_r1; ++k2) {
        int r2 = (k2 == 0) ? r1 : nbr[nbr_ptr[r1 - 1] + k2 - 2];
        if (r2 == 0) continue;
        if (r2 < 0) { delete op; return fail("build_augcls_operator: the closure reaches the edge of the site cluster"); }
        int sites[3], nsit = 1;
        sites[0] = r;
        if (r1 != r) sites[nsit++] = r1;
        if (r2 != r && r2 != r1) sites[nsit++] = r2;
        int ncomb = 1;
        for (int j = 0; j < nsit; ++j) ncomb *= nst[sites[j] - 1];
        for (int f = 0; f < ncomb; ++f) {
          std::vector<int> cc = c0;
          int q = f;
          for (int j = 0; j < nsit; ++j) {
            int ns_ = nst[sites[j] - 1];
            if (ns_ == 1) continue;
            int dgt = q % ns_; q /= ns_;
            cc = set_state(cc, sites[j], dgt, nsm);
          }
          if ((int)cc.size() > rkmax) continue;
          canon_node(perm, n, nop, nsm, r2, cc, cs, ccf, osz, gb);
          int id = st.find_or_add(cs, ccf.data(), (int)ccf.size(), lev + 1, isnew);
          if (isnew) st.orb[id - 1] = osz;
        }
      }
    }
  }
  // ---- tables
  const int nn = st.n;
  op->nn = nn; op->nop = nop; op->nsmax = nsm; op->ncls = ncls; op->nsp = nsp;
  op->nsc.assign(nsc, nsc + ncls); op->ldspc = ldspc; op->spc.assign(spc, spc + (size_t)ldspc * ncls);
  op->mt.assign((size_t)nsm * nsm * nsm * ncls, 0.0);
  for (int kap = 0; kap < ncls; ++kap) {
    std::vector<double> cvec(conc + (size_t)ldspc * kap, conc + (size_t)ldspc * kap + nsc[kap]);
    class_mt(cvec, nsm, &op->mt[(size_t)nsm * nsm * nsm * kap]);
  }
  int ns = 0;
  for (int r = 0; r < n; ++r) ns = std::max(ns, nbr_ptr[r + 1] - nbr_ptr[r]);
  op->nslot = ns;
  op->flipr.assign((size_t)nsm * nn, 0); op->flipg.assign((size_t)nsm * nn, 1);
  op->hopr.assign((size_t)ns * nn, 0); op->hopg.assign((size_t)ns * nn, 1);
  op->lst.assign(nn, 0); op->site.assign(nn, 0); op->ncl.assign(nn, 0); op->frozen.assign(nn, 0); op->level.assign(nn, 0);
  op->norb.assign(nn, 0.0); op->sq.assign(nn, 0.0);
  op->c.assign(9 * (size_t)nsp, 0.0); op->d = op->c; op->o = op->c; op->e = op->c;
  op->block0.assign(81 * (size_t)nty, 0.0);
  if (block0) for (size_t q = 0; q < 81 * (size_t)nty; ++q) op->block0[q] = block0[q];
  op->pi.assign(9 * (size_t)nop, 0); op->sg.assign(9 * (size_t)nop, 0.0); op->chi.assign(nop, 1.0); op->csg.assign(9 * (size_t)nop, 0.0);
  op->dmat.assign(dmat, dmat + 81 * (size_t)nop);
  for (int g = 0; g < nop; ++g)
    for (int l = 0; l < 9; ++l) {
      op->pi[l + 9 * g] = 0; op->sg[l + 9 * g] = 0.0;
      for (int jj = 0; jj < 9; ++jj) {
        double v = dmat[jj + 9 * (l + 9 * (size_t)g)];
        if (std::fabs(v) > 0.5) { op->pi[l + 9 * g] = jj + 1; op->sg[l + 9 * g] = v; }
      }
      if (op->pi[l + 9 * g] == 0) { delete op; return fail("build_augcls_operator: orbital operation is not monomial"); }
    }
  if (nsb < ns) { delete op; return fail("build_augcls_operator: fewer bond blocks than neighbour slots"); }
  op->btab.assign((size_t)81 * ns * nop * nty, 0.0);
  for (int t = 0; t < nty; ++t)
    for (int g = 0; g < nop; ++g)
      for (int k = 0; k < ns; ++k)
        for (int l = 0; l < 9; ++l)
          for (int jj = 0; jj < 9; ++jj) {
            int l2 = op->pi[jj + 9 * g] - 1;
            size_t dst = l + 9 * (l2 + 9 * (k + (size_t)ns * (g + (size_t)nop * t)));
            op->btab[dst] = op->btab[dst] + block[l + 9 * (jj + 9 * (k + (size_t)nsb * t))] * op->sg[jj + 9 * g];
          }
  for (int g = 0; g < nop; ++g) { op->chi[g] = 1.0; for (int l = 0; l < 9; ++l) op->csg[l + 9 * g] = op->sg[l + 9 * g]; }
  op->stab_ptr.assign(nn + 1, 0);
  std::vector<int> nstb(nn, 0);
  for (int i = 0; i < nn; ++i) {
    int r = st.site[i];
    std::vector<int> c0(st.data.begin() + st.start[i], st.data.begin() + st.start[i] + st.len[i]);
    for (int g = 0; g < nop; ++g) {
      const int* p = perm + (size_t)g * n;
      if (p[r - 1] != r) continue;
      std::vector<int> c2(c0.size());
      for (size_t k = 0; k < c0.size(); ++k) c2[k] = p[c0[k] / nsm - 1] * nsm + c0[k] % nsm;
      sort_small(c2);
      if (c2 == c0) ++nstb[i];
    }
    if (nstb[i] * st.orb[i] != nop) { delete op; return fail("build_augcls_operator: stabiliser size /= group order / orbit size"); }
  }
  op->stab_ptr[0] = 1;
  for (int i = 0; i < nn; ++i) op->stab_ptr[i + 1] = op->stab_ptr[i] + nstb[i];
  op->stab.assign(op->stab_ptr[nn] - 1, 0);
  for (int i = 0; i < nn; ++i) {
    int r = st.site[i];
    std::vector<int> c0(st.data.begin() + st.start[i], st.data.begin() + st.start[i] + st.len[i]);
    int j = op->stab_ptr[i];
    for (int g = 0; g < nop; ++g) {
      const int* p = perm + (size_t)g * n;
      if (p[r - 1] != r) continue;
      std::vector<int> c2(c0.size());
      for (size_t k = 0; k < c0.size(); ++k) c2[k] = p[c0[k] / nsm - 1] * nsm + c0[k] % nsm;
      sort_small(c2);
      if (c2 == c0) { op->stab[j - 1] = g + 1; ++j; }
    }
    op->level[i] = st.level[i]; op->norb[i] = (double)st.orb[i]; op->sq[i] = std::sqrt(op->norb[i]); op->site[i] = r;
    op->ncl[i] = cls[r - 1];
    op->lst[i] = get_state(c0, r, nsm);
    for (int k = 0; k < nsc[cls[r - 1] - 1]; ++k) {
      if (k == op->lst[i]) { op->flipr[k + (size_t)nsm * i] = i + 1; op->flipg[k + (size_t)nsm * i] = 1; }
      else if (k == 0 || canflip[r - 1]) {
        std::vector<int> tmp = set_state(c0, r, k, nsm);
        canon_node(perm, n, nop, nsm, r, tmp, cs, ccf, osz, gb);
        int jj = st.find(cs, ccf.data(), (int)ccf.size());
        if (jj > 0) { op->flipr[k + (size_t)nsm * i] = jj; op->flipg[k + (size_t)nsm * i] = gb; }
      }
    }
    int deg = nbr_ptr[r] - nbr_ptr[r - 1];
    for (int k = 0; k < deg; ++k) {
      int nb = nbr[nbr_ptr[r - 1] + k - 1];
      if (nb <= 0) continue;
      canon_node(perm, n, nop, nsm, nb, c0, cs, ccf, osz, gb);
      int jj = st.find(cs, ccf.data(), (int)ccf.size());
      if (jj > 0) { op->hopr[k + (size_t)ns * i] = jj; op->hopg[k + (size_t)ns * i] = gb; }
    }
  }
  // target links (src/asr_augcls.f90:808-820): site r alone in local state k, every other site in its reference state
  for (int t = 0; tsite && t < ntarget; ++t) {
    int r = tsite[t];
    for (int k = 0; k < nsm; ++k) { tnode[k + (size_t)nsm * t] = 0; tgop[k + (size_t)nsm * t] = 1; }
    if (r < 1 || r > n) { delete op; return fail("build_augcls_operator: target site out of range"); }
    for (int k = 0; k < nsc[cls[r - 1] - 1]; ++k) {
      if (k > 0 && (r == start || !canflip[r - 1])) continue;
      std::vector<int> tmp = set_state(cfg0, r, k, nsm);
      canon_node(perm, n, nop, nsm, r, tmp, cs, ccf, osz, gb);
      tnode[k + (size_t)nsm * t] = st.find(cs, ccf.data(), (int)ccf.size());
      if (tnode[k + (size_t)nsm * t] < 0) tnode[k + (size_t)nsm * t] = 0;
      tgop[k + (size_t)nsm * t] = gb;
    }
  }
  *handle = op;
  return 0;
}
extern "C" int orc_build(int n, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc, int ldspc,
                         const double* conc, int nsp, const int* cls, const int* perm, int nop, const double* dmat,
                         int start, int maxlevel, int maxrank, const int* flippable, const int* stype,
                         const double* block, int nsb, int ntb, const double* block0, void** handle) {
  return build_impl(n, nbr_ptr, nbr, ncls, nsc, spc, ldspc, conc, nsp, cls, perm, nop, dmat, start, maxlevel, maxrank,
                    flippable, stype, block, nsb, ntb, block0, nullptr, 0, nullptr, nullptr, handle);
}
extern "C" int orc_build_targets(int n, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc,
                                 int ldspc, const double* conc, int nsp, const int* cls, const int* perm, int nop,
                                 const double* dmat, int start, int maxlevel, int maxrank, const int* flippable,
                                 const int* stype, const double* block, int nsb, int ntb, const double* block0,
                                 const int* tsite, int ntarget, int* tnode, int* tgop, void** handle) {
  return build_impl(n, nbr_ptr, nbr, ncls, nsc, spc, ldspc, conc, nsp, cls, perm, nop, dmat, start, maxlevel, maxrank,
                    flippable, stype, block, nsb, ntb, block0, tsite, ntarget, tnode, tgop, handle);
}

extern "C" void orc_free(void* h) { delete (Op*)h; }

// dims: nn, nslot, nsmax, nop, ncls, ntype, nstab
extern "C" void orc_dims(void* h, int* out) {
  Op* op = (Op*)h;
  out[0] = op->nn; out[1] = op->nslot; out[2] = op->nsmax; out[3] = op->nop; out[4] = op->ncls; out[5] = op->ntype;
  out[6] = op->stab_ptr[op->nn] - 1;
}

extern "C" void orc_tables(void* h, int* flipr, int* flipg, int* hopr, int* hopg, int* lst, int* site, int* ncl, int* level,
                           double* norb, double* sq, int* stab_ptr, int* stab, int* pi, double* sg, double* mt) {
  Op* op = (Op*)h;
  std::copy(op->flipr.begin(), op->flipr.end(), flipr); std::copy(op->flipg.begin(), op->flipg.end(), flipg);
  std::copy(op->hopr.begin(), op->hopr.end(), hopr); std::copy(op->hopg.begin(), op->hopg.end(), hopg);
  std::copy(op->lst.begin(), op->lst.end(), lst); std::copy(op->site.begin(), op->site.end(), site);
  std::copy(op->ncl.begin(), op->ncl.end(), ncl); std::copy(op->level.begin(), op->level.end(), level);
  std::copy(op->norb.begin(), op->norb.end(), norb); std::copy(op->sq.begin(), op->sq.end(), sq);
  std::copy(op->stab_ptr.begin(), op->stab_ptr.end(), stab_ptr); std::copy(op->stab.begin(), op->stab.end(), stab);
  std::copy(op->pi.begin(), op->pi.end(), pi); std::copy(op->sg.begin(), op->sg.end(), sg);
  std::copy(op->mt.begin(), op->mt.end(), mt);
}

// ---- parameter setters: src/asr_augcls.f90:107-185
extern "C" int orc_set_start(void* h, int l0) {              // augcls_set_start :107-118
  Op* op = (Op*)h;
  op->start_l = l0;
  for (int g = 0; g < op->nop; ++g) {
    double v = op->dmat[(l0 - 1) + 9 * ((l0 - 1) + 9 * (size_t)g)];
    if (std::fabs(std::fabs(v) - 1.0) > 1.0e-9) return fail("augcls_set_start: start orbital is not one-dimensional under the group");
    op->chi[g] = v >= 0 ? 1.0 : -1.0;
    for (int l = 0; l < 9; ++l) op->csg[l + 9 * g] = op->chi[g] * op->sg[l + 9 * g];
  }
  return 0;
}
extern "C" int orc_set_chi(void* h, const double* chi) {     // augcls_set_chi :165-174
  Op* op = (Op*)h;
  for (int g = 0; g < op->nop; ++g) {
    op->chi[g] = chi[g];
    for (int l = 0; l < 9; ++l) op->csg[l + 9 * g] = op->chi[g] * op->sg[l + 9 * g];
  }
  return 0;
}
extern "C" void orc_set_params(void* h, const double* c, const double* d, const double* o, const double* e) {   // :121-126
  Op* op = (Op*)h;
  size_t m = 9 * (size_t)op->nsp;
  op->c.assign(c, c + m); op->d.assign(d, d + m); op->o.assign(o, o + m); op->e.assign(e, e + m);
}
// the node loop shared by augcls_freeze_site and augcls_freeze_any: every node of the site must sit on a site that was not
// flippable (own state 0, at most one flip link)
static int freeze_nodes(Op* op, int site, int sp, const char* who, int* nfound) {
  int n = 0;
  for (int i = 0; i < op->nn; ++i) {   // the reference stops at the first flippable node; nothing is changed before it here
    if (op->site[i] != site) continue;
    int nz = 0;
    for (int k = 0; k < op->nsmax; ++k) if (op->flipr[k + (size_t)op->nsmax * i] != 0) ++nz;
    if (op->lst[i] != 0 || nz > 1) return fail((std::string(who) + ": the frozen site was flippable").c_str());
    ++n;
  }
  for (int i = 0; i < op->nn; ++i)
    if (op->site[i] == site) op->frozen[i] = sp;
  if (nfound) *nfound = n;
  return 0;
}
// augcls_freeze_site :129-142: the species must belong to the class of the start node when the site is the start site
extern "C" int orc_freeze_site(void* h, int site, int sp) {
  Op* op = (Op*)h;
  if (sp < 1 || sp > op->nsp) return fail("augcls_freeze_site: species index out of range");
  if (op->site[0] == site) {
    const int kap = op->ncl[0] - 1;
    bool in = false;
    for (int k = 0; k < op->nsc[kap]; ++k) if (op->spcv(k, kap) == sp) in = true;
    if (!in) return fail("augcls_freeze_site: species not in the class of the frozen site");
  }
  return freeze_nodes(op, site, sp, "augcls_freeze_site", nullptr);
}
// augcls_freeze_any :147-161: any species index 1..nsp; nfound = nodes on the site
extern "C" int orc_freeze_any(void* h, int site, int sp, int* nfound) {
  Op* op = (Op*)h;
  if (sp < 1 || sp > op->nsp) return fail("augcls_freeze_any: species index out of range");
  return freeze_nodes(op, site, sp, "augcls_freeze_any", nfound);
}
extern "C" void orc_unfreeze(void* h) { Op* op = (Op*)h; std::fill(op->frozen.begin(), op->frozen.end(), 0); }
extern "C" int orc_set_class_conc(void* h, int kap, const double* conc) {   // augcls_set_class_conc :178-185
  Op* op = (Op*)h;
  int nsc = op->nsc[kap - 1];
  double s = 0.0;
  for (int k = 0; k < nsc; ++k) { if (conc[k] < 0.0) return fail("augcls_set_class_conc: concentrations"); s += conc[k]; }
  if (std::fabs(s - 1.0) > 1.0e-8) return fail("augcls_set_class_conc: concentrations");
  std::vector<double> cv(conc, conc + nsc);
  int nsm = op->nsmax;
  class_mt(cv, nsm, &op->mt[(size_t)nsm * nsm * nsm * (kap - 1)]);
  return 0;
}
extern "C" void orc_set_stype_blocks(void* h, const int* stype) {
  Op* op = (Op*)h;
  for (int i = 0; i < op->nsite; ++i) op->stype[i] = stype[i];
}

// ===================================================================================================== application
// local_weights src/asr_augcls.f90:362-377: wt(lam, k, kk, kap) = sum_s par(lam, spc(s)) mt(k, kk, s, kap)
static void local_weights(const Op& op, const double* par, std::vector<double>& wt) {
  int nsm = op.nsmax;
  wt.assign((size_t)9 * nsm * nsm * op.ncls, 0.0);
  for (int kap = 0; kap < op.ncls; ++kap)
    for (int kk = 0; kk < op.nsc[kap]; ++kk)
      for (int k = 0; k < op.nsc[kap]; ++k)
        for (int s = 0; s < op.nsc[kap]; ++s)
          for (int lam = 0; lam < 9; ++lam) {
            size_t w = lam + 9 * (k + (size_t)nsm * (kk + (size_t)nsm * kap));
            wt[w] = wt[w] + par[lam + 9 * (size_t)(op.spcv(s, kap) - 1)] * op.mt[k + nsm * (kk + nsm * (s + (size_t)nsm * kap))];
          }
}
#define WT(w, lam, k, kk, kap) (w)[(lam) + 9 * ((k) + (size_t)nsm * ((kk) + (size_t)nsm * (kap)))]

// Threads of the node loops of one operator application, for large parity cases in the tests: 1 unless the caller sets
// more, and always serial inside an enclosing parallel region (chain_greens' tasks).  Every output node is computed by
// one thread with the same operations in the same order, so the results are the same bits for every thread count.
static int g_apply_threads = 1;
extern "C" void orc_set_apply_threads(int n) { g_apply_threads = n < 1 ? 1 : n; }
extern "C" int orc_apply_threads() { return g_apply_threads; }
#define ORC_NODE_LOOP _Pragma("omp parallel for schedule(static) num_threads(g_apply_threads) if (g_apply_threads > 1 && !omp_in_parallel())")

// apply_rand src/asr_augcls.f90:380-403 (amplitude coordinates)
static void apply_rand(const Op& op, const double* par, const double* x, double* w) {
  std::vector<double> wt;
  local_weights(op, par, wt);
  const int nsm = op.nsmax;
  ORC_NODE_LOOP
  for (int i = 0; i < op.nn; ++i) {
    const double* xi = x + 9 * (size_t)i;
    double* wi = w + 9 * (size_t)i;
    if (op.frozen[i] > 0) {
      for (int l = 0; l < 9; ++l) wi[l] = par[l + 9 * (size_t)(op.frozen[i] - 1)] * xi[l];
      continue;
    }
    int kap = op.ncl[i] - 1, l0 = op.lst[i];
    double acc[9];
    for (int l = 0; l < 9; ++l) acc[l] = WT(wt, l, l0, l0, kap) * xi[l];
    for (int k = 0; k < op.nsc[kap]; ++k) {
      int r = op.flipr[k + (size_t)nsm * i];
      if (k == l0 || r == 0) continue;
      int g = op.flipg[k + (size_t)nsm * i] - 1;
      for (int l = 0; l < 9; ++l) {
        double tf = op.csg[l + 9 * g] * x[9 * (size_t)(r - 1) + op.pi[l + 9 * g] - 1];
        acc[l] = acc[l] + WT(wt, l, l0, k, kap) * tf;
      }
    }
    for (int l = 0; l < 9; ++l) wi[l] = acc[l];
  }
}

// apply_h src/asr_augcls.f90:449-489: hx = c x + D S D x (amplitude coordinates)
static void apply_h(const Op& op, const double* x, double* hx, double* t1, double* t2, double* t3) {
  apply_rand(op, op.d.data(), x, t1);
  const int ns = op.nslot, nop = op.nop;
  ORC_NODE_LOOP
  for (int i = 0; i < op.nn; ++i) {
    int t = op.stype[op.site[i] - 1] - 1;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int l2 = 0; l2 < 9; ++l2) {
      double tl = t1[9 * (size_t)i + l2];
      for (int l = 0; l < 9; ++l) acc[l] = acc[l] + op.block0[l + 9 * (l2 + 9 * (size_t)t)] * tl;
    }
    for (int k = 0; k < ns; ++k) {
      int r = op.hopr[k + (size_t)ns * i];
      if (r == 0) continue;
      int g = op.hopg[k + (size_t)ns * i] - 1;
      for (int l2 = 0; l2 < 9; ++l2) {
        double tl = op.chi[g] * t1[9 * (size_t)(r - 1) + l2];
        const double* bt = &op.btab[9 * (l2 + 9 * (k + (size_t)ns * (g + (size_t)nop * t)))];
        for (int l = 0; l < 9; ++l) acc[l] = acc[l] + bt[l] * tl;
      }
    }
    for (int l = 0; l < 9; ++l) t2[9 * (size_t)i + l] = acc[l];
  }
  apply_rand(op, op.d.data(), t2, t3);
  apply_rand(op, op.c.data(), x, hx);
  const long nd = 9 * (long)op.nn;
  ORC_NODE_LOOP
  for (long q = 0; q < nd; ++q) hx[q] = hx[q] + t3[q];
}

// augcls_apply src/asr_augcls.f90:275-297: y = H x in normalised coordinates, H = E_nu + h - h o h
struct Work { std::vector<double> w[8]; void init(size_t n) { for (auto& v : w) v.assign(n, 0.0); } };
static void augcls_apply(const Op& op, Work& wk, const double* x, double* y) {
  size_t nd = 9 * (size_t)op.nn;
  if (wk.w[0].size() != nd) wk.init(nd);
  ORC_NODE_LOOP
  for (int i = 0; i < op.nn; ++i)
    for (int l = 0; l < 9; ++l) wk.w[6][9 * (size_t)i + l] = x[9 * (size_t)i + l] / op.sq[i];
  apply_h(op, wk.w[6].data(), wk.w[0].data(), wk.w[3].data(), wk.w[4].data(), wk.w[5].data());
  apply_rand(op, op.o.data(), wk.w[0].data(), wk.w[1].data());
  apply_h(op, wk.w[1].data(), wk.w[2].data(), wk.w[3].data(), wk.w[4].data(), wk.w[5].data());
  apply_rand(op, op.e.data(), wk.w[6].data(), wk.w[7].data());
  ORC_NODE_LOOP
  for (int i = 0; i < op.nn; ++i)
    for (int l = 0; l < 9; ++l) {
      size_t q = 9 * (size_t)i + l;
      y[q] = op.sq[i] * (wk.w[7][q] + wk.w[0][q] - wk.w[2][q]);
    }
}
extern "C" void orc_apply(void* h, const double* x, double* y) {
  Op* op = (Op*)h;
  Work wk;
  augcls_apply(*op, wk, x, y);
}

// augcls_rand_c src/asr_augcls.f90:419-446: w = X x, complex parameters par(9, nsp), normalised coordinates
static void augcls_rand_c(const Op& op, const cd* par, const cd* x, cd* w) {
  std::vector<double> pr(9 * (size_t)op.nsp), pim(9 * (size_t)op.nsp);
  for (size_t q = 0; q < pr.size(); ++q) { pr[q] = par[q].real(); pim[q] = par[q].imag(); }
  std::vector<double> wr, wi;
  local_weights(op, pr.data(), wr);
  local_weights(op, pim.data(), wi);
  const int nsm = op.nsmax;
  for (int i = 0; i < op.nn; ++i) {
    cd xi[9];
    for (int l = 0; l < 9; ++l) xi[l] = x[9 * (size_t)i + l] / op.sq[i];
    if (op.frozen[i] > 0) {
      for (int l = 0; l < 9; ++l) w[9 * (size_t)i + l] = par[l + 9 * (size_t)(op.frozen[i] - 1)] * x[9 * (size_t)i + l];
      continue;
    }
    int kap = op.ncl[i] - 1, l0 = op.lst[i];
    cd acc[9];
    for (int l = 0; l < 9; ++l) acc[l] = cd(WT(wr, l, l0, l0, kap), WT(wi, l, l0, l0, kap)) * xi[l];
    for (int k = 0; k < op.nsc[kap]; ++k) {
      int r = op.flipr[k + (size_t)nsm * i];
      if (k == l0 || r == 0) continue;
      int g = op.flipg[k + (size_t)nsm * i] - 1;
      for (int l = 0; l < 9; ++l) {
        cd tf = op.csg[l + 9 * g] * x[9 * (size_t)(r - 1) + op.pi[l + 9 * g] - 1];
        tf = tf / op.sq[r - 1];
        acc[l] = acc[l] + cd(WT(wr, l, l0, k, kap), WT(wi, l, l0, k, kap)) * tf;
      }
    }
    for (int l = 0; l < 9; ++l) w[9 * (size_t)i + l] = op.sq[i] * acc[l];
  }
}
extern "C" void orc_rand_c(void* h, const double* par /* complex (9,nsp) interleaved */, const double* x, double* w) {
  augcls_rand_c(*(Op*)h, (const cd*)par, (const cd*)x, (cd*)w);
}

// augcls_project_c src/asr_augcls.f90:329-348
static void augcls_project_c(const Op& op, cd* x) {
  for (int i = 0; i < op.nn; ++i) {
    int ns = op.stab_ptr[i + 1] - op.stab_ptr[i];
    if (ns <= 1) continue;
    cd acc[9];
    for (int j = op.stab_ptr[i]; j < op.stab_ptr[i + 1]; ++j) {
      int g = op.stab[j - 1] - 1;
      for (int l = 0; l < 9; ++l) acc[l] = acc[l] + op.csg[l + 9 * g] * x[9 * (size_t)i + op.pi[l + 9 * g] - 1];
    }
    for (int l = 0; l < 9; ++l) x[9 * (size_t)i + l] = acc[l] / (double)ns;
  }
}
extern "C" void orc_project_c(void* h, double* x) { augcls_project_c(*(Op*)h, (cd*)x); }

// augcls_hp_c src/asr_augcls.f90:301-320: y = h x, complex, normalised coordinates
static void hp_c(const Op& op, const cd* x, cd* y) {
  size_t nd = 9 * (size_t)op.nn;
  std::vector<double> a(nd), b(nd), h1(nd), h2(nd), t1(nd), t2(nd), t3(nd);
  for (int i = 0; i < op.nn; ++i)
    for (int l = 0; l < 9; ++l) {
      size_t q = 9 * (size_t)i + l;
      a[q] = x[q].real() / op.sq[i]; b[q] = x[q].imag() / op.sq[i];
    }
  apply_h(op, a.data(), h1.data(), t1.data(), t2.data(), t3.data());
  apply_h(op, b.data(), h2.data(), t1.data(), t2.data(), t3.data());
  for (int i = 0; i < op.nn; ++i)
    for (int l = 0; l < 9; ++l) { size_t q = 9 * (size_t)i + l; y[q] = op.sq[i] * cd(h1[q], h2[q]); }
}
extern "C" void orc_hp_c(void* h, const double* xin, double* yout) { hp_c(*(Op*)h, (const cd*)xin, (cd*)yout); }

// ===================================================================================================== eigenvalues
// Eigenvalues of a complex upper-Hessenberg matrix (here: the complex-symmetric tridiagonal chain matrix) by the
// single-shift QR algorithm with unitary Givens rotations, Wilkinson shifts and exceptional shifts (Golub & Van Loan,
// Matrix Computations, 4th ed., Alg. 7.5.1 / the EISPACK COMQR scheme).  Stands in for LAPACK zgeev(JOBVL=JOBVR='N').
static int hess_eigvals(int n, std::vector<cd>& H /* row-major n x n */, cd* ev) {
  auto A = [&](int i, int j) -> cd& { return H[(size_t)i * n + j]; };
  int hi = n - 1, iter = 0, total = 0;
  while (hi >= 0) {
    if (hi == 0) { ev[0] = A(0, 0); break; }
    int l = hi;
    while (l > 0) {
      double s = std::abs(A(l - 1, l - 1)) + std::abs(A(l, l));
      if (s == 0.0) s = 1.0;
      if (std::abs(A(l, l - 1)) <= DBL_EPSILON * s) { A(l, l - 1) = 0.0; break; }
      --l;
    }
    if (l == hi) { ev[hi] = A(hi, hi); --hi; iter = 0; continue; }
    ++iter; ++total;
    if (total > 60 * n) return 1;
    cd mu;
    if (iter == 10 || iter == 20) {
      mu = A(hi, hi) + std::fabs(A(hi, hi - 1).real()) + (hi >= 2 ? std::fabs(A(hi - 1, hi - 2).real()) : 0.0);
    } else {
      cd a = A(hi - 1, hi - 1), b = A(hi - 1, hi), c = A(hi, hi - 1), d = A(hi, hi);
      cd tr2 = 0.5 * (a + d), det = a * d - b * c;
      cd disc = std::sqrt(tr2 * tr2 - det);
      cd m1 = tr2 + disc, m2 = tr2 - disc;
      mu = (std::abs(m1 - d) <= std::abs(m2 - d)) ? m1 : m2;
    }
    for (int k = l; k <= hi; ++k) A(k, k) -= mu;
    std::vector<cd> cs(hi - l), sn(hi - l);
    for (int k = l; k < hi; ++k) {
      cd x = A(k, k), y = A(k + 1, k);
      double r = std::hypot(std::abs(x), std::abs(y));
      cd c = 1.0, s = 0.0;
      if (r > 0.0) { c = x / r; s = y / r; }
      cs[k - l] = c; sn[k - l] = s;
      for (int j = k; j <= hi; ++j) {
        cd u = A(k, j), v = A(k + 1, j);
        A(k, j) = std::conj(c) * u + std::conj(s) * v;
        A(k + 1, j) = -s * u + c * v;
      }
    }
    for (int k = l; k < hi; ++k) {
      cd c = cs[k - l], s = sn[k - l];
      int rmax = std::min(k + 2, hi);
      for (int i = l; i <= rmax; ++i) {
        cd u = A(i, k), v = A(i, k + 1);
        A(i, k) = c * u + s * v;
        A(i, k + 1) = -std::conj(s) * u + std::conj(c) * v;
      }
    }
    for (int k = l; k <= hi; ++k) A(k, k) += mu;
  }
  return 0;
}
static int chain_eigvals(int m, const cd* a, const cd* b, cd am, cd* ev) {
  std::vector<cd> H((size_t)m * m, 0.0);
  for (int j = 0; j < m; ++j) {
    H[(size_t)j * m + j] = a[j];
    if (j < m - 1) { H[(size_t)j * m + j + 1] = b[j]; H[(size_t)(j + 1) * m + j] = b[j]; }
  }
  H[(size_t)(m - 1) * m + m - 1] = am;
  return hess_eigvals(m, H, ev);
}
extern "C" int orc_chain_eigvals(int m, const double* a, const double* b, double* ev) {
  return chain_eigvals(m, (const cd*)a, (const cd*)b, ((const cd*)a)[m - 1], (cd*)ev);
}

// ===================================================================================================== continued fraction
// cf_species src/asr_chain.f90:67-167.  tail: 0 none, 1 hull, 2 bp, 3 avg2.  nfall (optional) counts bp fallbacks.
static int minloc_re(int m, const cd* ev) { int k = 0; for (int j = 1; j < m; ++j) if (ev[j].real() < ev[k].real()) k = j; return k; }
static int maxloc_re(int m, const cd* ev) { int k = 0; for (int j = 1; j < m; ++j) if (ev[j].real() > ev[k].real()) k = j; return k; }

static void cf_species(const cd* a, const cd* b, const cd* c, int m, cd z, int tail, cd& g11, cd& f, cd* edges, cd* pv,
                       long* nfall) {
  cd aa, bb;
  int info = 1;
  std::vector<cd> ev(std::max(m, 1));
  if (m >= 2 && tail != 0) info = chain_eigvals(m, a, b, a[m - 1], ev.data());
  if (info == 0) {
    int ilo = minloc_re(m, ev.data()), ihi = maxloc_re(m, ev.data());
    aa = 0.5 * (ev[ilo] + ev[ihi]); bb = 0.25 * (ev[ihi] - ev[ilo]);
    if (tail == 2) {   // bp_fixed_point :126-156
      bool done = false;
      for (int it = 0; it < 200 && !done; ++it) {
        if (chain_eigvals(m, a, b, a[m - 1] + bb, ev.data())) { if (nfall) ++*nfall; done = true; break; }
        cd ep = ev[maxloc_re(m, ev.data())];
        if (chain_eigvals(m, a, b, a[m - 1] - bb, ev.data())) { if (nfall) ++*nfall; done = true; break; }
        cd em = ev[minloc_re(m, ev.data())];
        cd an = 0.5 * (ep + em), bn = 0.25 * (ep - em);
        if (std::abs(an - aa) + std::abs(bn - bb) < 1.0e-12 * (1.0 + std::abs(bn))) { aa = an; bb = bn; done = true; break; }
        aa = an; bb = bn;
      }
      if (!done) {
        if (nfall) ++*nfall;
        chain_eigvals(m, a, b, a[m - 1], ev.data());
        int ilo2 = minloc_re(m, ev.data()), ihi2 = maxloc_re(m, ev.data());
        aa = 0.5 * (ev[ilo2] + ev[ihi2]); bb = 0.25 * (ev[ihi2] - ev[ilo2]);
      }
    }
  } else {
    aa = a[m - 1]; bb = 0.0;
    if (m > 1) bb = b[m - 2];
  }
  if (tail == 3 && m >= 3) { aa = 0.5 * (a[m - 1] + a[m - 2]); bb = std::sqrt(0.5 * (b[m - 2] * b[m - 2] + b[m - 3] * b[m - 3])); }
  if (tail == 0) { aa = 0.0; bb = 0.0; }
  if (edges) { edges[0] = aa; edges[1] = bb; }
  cd d = z - aa, tl;
  if (std::abs(bb) < 1.0e-14) tl = 0.0;
  else {
    cd s = std::sqrt(d * d - 4.0 * bb * bb);
    cd g1 = (d - s) / (2.0 * bb * bb), g2 = (d + s) / (2.0 * bb * bb);
    tl = (std::abs(bb * g1) <= std::abs(bb * g2)) ? bb * bb * g1 : bb * bb * g2;
  }
  std::vector<cd> gt(m + 1);
  gt[m] = 0.0;
  gt[m - 1] = 1.0 / (z - a[m - 1] - tl);
  for (int j = m - 2; j >= 0; --j) gt[j] = 1.0 / (z - a[j] - b[j] * b[j] * gt[j + 1]);
  g11 = gt[0];
  f = 0.0;
  cd prod = gt[0];
  for (int k = 0; k < m; ++k) {
    if (c) f = f + c[k] * prod;
    if (pv) pv[k] = prod;
    if (k < m - 1) prod = prod * b[k] * gt[k + 1];
  }
}
extern "C" void orc_cf_species(const double* a, const double* b, const double* c, int m, double zr, double zi, int tail,
                               double* g, double* f, double* edges, double* pv, long* nfall) {
  cd g11, ff;
  cf_species((const cd*)a, (const cd*)b, (const cd*)c, m, cd(zr, zi), tail, g11, ff, (cd*)edges, (cd*)pv, nfall);
  g[0] = g11.real(); g[1] = g11.imag();
  if (f) { f[0] = ff.real(); f[1] = ff.imag(); }
}

// ---- real chains: src/reference/asr_greens.f90 and asr_terminator.f90
// sqrt_tail asr_greens.f90:12-22
static cd sqrt_tail(cd z, double ainf, double binf) {
  cd w = z - ainf;
  cd s = std::sqrt(w * w - 4.0 * binf * binf);
  cd g1 = (w - s) / (2.0 * binf * binf), g2 = (w + s) / (2.0 * binf * binf);
  cd g = (std::abs(g1) <= std::abs(g2)) ? g1 : g2;
  return binf * binf * g;
}
// periodic_g asr_greens.f90:30-58
static cd periodic_g(cd z, const double* ap, const double* bp, int p) {
  cd m[2][2] = {{1.0, 0.0}, {0.0, 1.0}};
  for (int k = 0; k < p; ++k) {
    cd mk[2][2] = {{0.0, 1.0}, {-bp[k] * bp[k], z - ap[k]}};
    cd t[2][2];
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) t[i][j] = m[i][0] * mk[0][j] + m[i][1] * mk[1][j];
    for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) m[i][j] = t[i][j];
  }
  cd tr = m[0][0] + m[1][1], det = m[0][0] * m[1][1] - m[0][1] * m[1][0];
  cd disc = std::sqrt(tr * tr - 4.0 * det);
  cd l1 = 0.5 * (tr + disc), l2 = 0.5 * (tr - disc);
  cd lam = (std::abs(l1) >= std::abs(l2)) ? l1 : l2;
  cd g;
  if (std::abs(m[0][1]) > 0.0 || std::abs(m[0][0] - lam) > 0.0) {
    if (std::abs(lam - m[0][0]) > std::abs(m[1][0])) g = m[0][1] / (lam - m[0][0]);
    else g = (lam - m[1][1]) / m[1][0];
  } else g = (lam - m[1][1]) / m[1][0];
  return g;
}
// cf_green asr_greens.f90:80-90
static cd cf_green(const double* a, const double* b, int n, cd z, cd tl) {
  cd g = 1.0 / (z - a[n - 1] - tl);
  for (int i = n - 2; i >= 0; --i) g = 1.0 / (z - a[i] - b[i] * b[i] * g);
  return g;
}
// extreme eigenvalue of a real symmetric tridiagonal (stands in for dsterf, asr_terminator.f90:76): Sturm bisection
static int sturm_count(int n, const double* d, const double* e, double x) {
  int cnt = 0;
  double q = d[0] - x;
  if (q < 0) ++cnt;
  for (int i = 1; i < n; ++i) {
    if (q == 0.0) q = DBL_EPSILON * (std::fabs(e[i - 1]) + DBL_MIN);
    q = d[i] - x - e[i - 1] * e[i - 1] / q;
    if (q < 0) ++cnt;
  }
  return cnt;
}
static double tridiag_extreme(int n, const double* d, const double* e, bool upper) {
  double lo = d[0], hi = d[0];
  for (int i = 0; i < n; ++i) {
    double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i < n - 1 ? std::fabs(e[i]) : 0.0);
    lo = std::min(lo, d[i] - r); hi = std::max(hi, d[i] + r);
  }
  double span = hi - lo;
  lo -= 1e-12 * (span + 1.0); hi += 1e-12 * (span + 1.0);
  int target = upper ? n : 1;   // smallest x with count(<x) >= target... bisection on count
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    int c = sturm_count(n, d, e, mid);
    if (c >= target) hi = mid; else lo = mid;
  }
  return 0.5 * (lo + hi);
}
// bp_asymptote asr_terminator.f90:39-67
extern "C" int orc_bp_asymptote(const double* a, const double* b, int n, double* ainf, double* binf, int* niter) {
  double A = 0.5 * (a[n - 1] + a[n - 2]);
  double B = std::sqrt(0.5 * (b[n - 1] * b[n - 1] + b[n - 2] * b[n - 2]));
  std::vector<double> d(n), e(std::max(n - 1, 1));
  int ok = 0, it;
  for (it = 1; it <= 500; ++it) {
    for (int i = 0; i < n; ++i) d[i] = a[i];
    for (int i = 0; i < n - 1; ++i) e[i] = b[i];
    d[n - 1] = a[n - 1] + B;
    double ep = tridiag_extreme(n, d.data(), e.data(), true);
    d[n - 1] = a[n - 1] - B;
    double em = tridiag_extreme(n, d.data(), e.data(), false);
    double an = 0.5 * (ep + em), bn = 0.25 * (ep - em);
    if (std::fabs(an - A) + std::fabs(bn - B) < 1.0e-13) { A = an; B = bn; ok = 1; break; }
    A = an; B = bn;
  }
  *ainf = A; *binf = B;
  if (niter) *niter = it;
  return ok;
}
extern "C" double orc_tridiag_extreme(int n, const double* d, const double* e, int upper) {
  return tridiag_extreme(n, d, e, upper != 0);
}
// make_terminator + terminated_green asr_terminator.f90:83-126.  method: 0 sqrt-last, 1 sqrt-avg2, 2 beer-pettifor,
// 3 periodic2; join: 0 butt, 1 luchini-nex.  Returns G at nz energies.
extern "C" int orc_terminated_green(const double* a, const double* b, int n, int method, int join, int ninterp,
                                    const double* z, int nz, double* g, double* tparams /* ainf, binf, ntot */) {
  double ainf = 0, binf = 0;
  int period = 1;
  double ap[2] = {0, 0}, bp[2] = {0, 0}, blink = 0;
  switch (method) {
    case 0: ainf = a[n - 1]; binf = b[n - 1]; break;
    case 1: ainf = 0.5 * (a[n - 1] + a[n - 2]); binf = std::sqrt(0.5 * (b[n - 1] * b[n - 1] + b[n - 2] * b[n - 2])); break;
    case 2: orc_bp_asymptote(a, b, n, &ainf, &binf, nullptr); break;
    case 3:
      period = 2; ap[0] = a[n - 2]; ap[1] = a[n - 1]; bp[0] = b[n - 2]; bp[1] = b[n - 1]; blink = b[n - 1];
      ainf = 0.5 * (a[n - 1] + a[n - 2]); binf = std::sqrt(0.5 * (b[n - 1] * b[n - 1] + b[n - 2] * b[n - 2]));
      break;
    default: return fail("make_terminator: unknown method");
  }
  int ni = (join == 1 && period == 1) ? ninterp : 0;
  int nt = n + ni;
  std::vector<double> ta(nt), tb(nt);
  for (int k = 0; k < n; ++k) { ta[k] = a[k]; tb[k] = b[k]; }
  for (int k = 1; k <= ni; ++k) {
    double f = (double)k / (double)(ni + 1);
    ta[n + k - 1] = a[n - 1] + f * (ainf - a[n - 1]);
    tb[n + k - 1] = b[n - 1] + f * (binf - b[n - 1]);
  }
  if (tparams) { tparams[0] = ainf; tparams[1] = binf; tparams[2] = nt; }
  for (int j = 0; j < nz; ++j) {
    cd zz(z[2 * j], z[2 * j + 1]), gg;
    if (period == 1) gg = cf_green(ta.data(), tb.data(), nt, zz, sqrt_tail(zz, ainf, binf));
    else gg = cf_green(ta.data(), tb.data(), nt, zz, blink * blink * periodic_g(zz, ap, bp, 2));
    g[2 * j] = gg.real(); g[2 * j + 1] = gg.imag();
  }
  return 0;
}
extern "C" void orc_terminator_coefs(const double* a, const double* b, int n, int ninterp, double ainf, double binf,
                                     double* ta, double* tb) {
  for (int k = 0; k < n; ++k) { ta[k] = a[k]; tb[k] = b[k]; }
  for (int k = 1; k <= ninterp; ++k) {
    double f = (double)k / (double)(ninterp + 1);
    ta[n + k - 1] = a[n - 1] + f * (ainf - a[n - 1]);
    tb[n + k - 1] = b[n - 1] + f * (binf - b[n - 1]);
  }
}
extern "C" void orc_sqrt_tail(double zr, double zi, double ainf, double binf, double* t) {
  cd v = sqrt_tail(cd(zr, zi), ainf, binf); t[0] = v.real(); t[1] = v.imag();
}
extern "C" void orc_periodic_g(double zr, double zi, const double* ap, const double* bp, int p, double* g) {
  cd v = periodic_g(cd(zr, zi), ap, bp, p); g[0] = v.real(); g[1] = v.imag();
}

// ===================================================================================================== chains
// lanczos src/reference/asr_recursion.f90:17-58 (plain real chain on augcls_apply, no reorthogonalisation)
extern "C" int orc_lanczos(void* h, const double* v0, int nmax, double tiny, double* a, double* b, int* nout) {
  Op& op = *(Op*)h;
  size_t nd = 9 * (size_t)op.nn;
  std::vector<double> u(nd), up(nd, 0.0), w(nd);
  Work wk;
  for (int i = 0; i < nmax; ++i) { a[i] = 0.0; b[i] = 0.0; }
  double nrm = 0.0;
  for (size_t q = 0; q < nd; ++q) nrm += v0[q] * v0[q];
  nrm = std::sqrt(nrm);
  for (size_t q = 0; q < nd; ++q) u[q] = v0[q] / nrm;
  double bn = 0.0;
  int n = 0;
  for (int i = 0; i < nmax; ++i) {
    augcls_apply(op, wk, u.data(), w.data());
    double s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += u[q] * w[q];
    a[i] = s;
    for (size_t q = 0; q < nd; ++q) w[q] = w[q] - a[i] * u[q] - bn * up[q];
    n = i + 1;
    s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += w[q] * w[q];
    bn = std::sqrt(s);
    if (i == nmax - 1) break;
    b[i] = bn;
    if (bn < tiny) break;
    up = u;
    for (size_t q = 0; q < nd; ++q) u[q] = w[q] / bn;
  }
  if (n == nmax) b[nmax - 1] = bn;
  *nout = n;
  return 0;
}

// Energy-dependent chain parameters (asr_edc edn_t): dc(9), del(9, ns), enu(9, ns)
struct Edn { int ns; std::vector<double> dc, del, enu; };

// edc_green src/asr_edc.f90:75-164 (single energy).  Optionally a, b (complex, nlev), mused.
static void edc_green(Op& op, const Edn& ed, cd z, int iv, int nlev, double depth_tol, int tail, bool project,
                      cd& g, cd* acoef, cd* bcoef, int* mused, long* nfall) {
  size_t nd = 9 * (size_t)op.nn;
  std::vector<cd> ep(9 * (size_t)ed.ns);
  for (int s = 0; s < ed.ns; ++s)
    for (int l = 0; l < 9; ++l) ep[l + 9 * s] = z - ed.dc[l] * (z - ed.enu[l + 9 * s]) / ed.del[l + 9 * s];
  std::vector<cd> u(nd, 0.0), up(nd, 0.0), w(nd), dg(nd);
  std::vector<double> re(nd), im(nd), sre(nd), sim(nd);
  u[iv - 1] = 1.0;
  std::vector<cd> a(nlev, 0.0), b(nlev, 0.0), cc(nlev, 0.0);
  int m = 0;
  cd gprev = 0.0, gtry, ftmp;
  Work wk;
  for (int k = 1; k <= nlev; ++k) {
    for (size_t q = 0; q < nd; ++q) { re[q] = u[q].real(); im[q] = u[q].imag(); }
    augcls_apply(op, wk, re.data(), sre.data());
    augcls_apply(op, wk, im.data(), sim.data());
    augcls_rand_c(op, ep.data(), u.data(), dg.data());
    for (size_t q = 0; q < nd; ++q) w[q] = cd(sre[q], sim[q]) + dg[q];
    cd s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += u[q] * w[q];
    a[k - 1] = s;
    m = k;
    if (k == nlev) break;
    if (depth_tol > 0.0 && k >= 8 && k % 4 == 0) {
      cf_species(a.data(), b.data(), cc.data(), k, z, tail, gtry, ftmp, nullptr, nullptr, nfall);
      if (k > 8 && std::abs(gtry - gprev) <= depth_tol * std::abs(gtry)) break;
      gprev = gtry;
    }
    cd ak = a[k - 1], bk = 0.0;
    if (k > 1) bk = b[k - 2];
    for (size_t q = 0; q < nd; ++q) {
      w[q] = w[q] - ak * u[q];
      if (k > 1) w[q] = w[q] - bk * up[q];
    }
    if (project) augcls_project_c(op, w.data());
    s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += w[q] * w[q];
    b[k - 1] = std::sqrt(s);
    if (std::abs(b[k - 1]) < 1.0e-12) break;
    bk = b[k - 1];
    for (size_t q = 0; q < nd; ++q) { up[q] = u[q]; u[q] = w[q] / bk; }
  }
  cd ff;
  cf_species(a.data(), b.data(), cc.data(), m, z, tail, g, ff, nullptr, nullptr, nfall);
  if (acoef) for (int k = 0; k < m; ++k) acoef[k] = a[k];
  if (bcoef) for (int k = 0; k < m; ++k) bcoef[k] = b[k];
  if (mused) *mused = m;
}
extern "C" void orc_edc_green(void* h, int ns, const double* dc, const double* del, const double* enu, double zr, double zi,
                              int iv, int nlev, double depth_tol, int tail, int project, double* g, double* a, double* b,
                              int* mused, long* nfall) {
  Edn ed{ns, std::vector<double>(dc, dc + 9), std::vector<double>(del, del + 9 * ns), std::vector<double>(enu, enu + 9 * ns)};
  cd gg;
  edc_green(*(Op*)h, ed, cd(zr, zi), iv, nlev, depth_tol, tail, project != 0, gg, (cd*)a, (cd*)b, mused, nfall);
  g[0] = gg.real(); g[1] = gg.imag();
}

// epi_start + epi_blocks src/asr_epi.f90:578-663 (with chain :588-636): s0 = v9 on node 1, |v> = h'|s0> (augcls_hp_c,
// projected), nv = sqrt(re(v . v)); chain from s0 with tv = v gives X0 and fa, chain from v / nv with tv = s0 gives
// X2 = nv^2 g and fb = nv f; x = (X0, (fa + fb) / 2, X2, fa - fb).  The operator's characters must be those of v9
// (orc_set_chi).  ed: dc (9), del, enu (9, ns).  mused: the two depths.
static void epi_chain(Op& op, const std::vector<cd>& ep, const std::vector<cd>& u0, const std::vector<cd>& tv, cd z, int nlev,
                      int tail, bool project, cd& g, cd& f, int& m) {
  size_t nd = 9 * (size_t)op.nn;
  std::vector<cd> u = u0, up(nd, 0.0), w(nd), dg(nd);
  std::vector<double> re(nd), im(nd), sre(nd), sim(nd);
  std::vector<cd> a(nlev, 0.0), b(nlev, 0.0), c(nlev, 0.0);
  Work wk;
  bool closed = false;
  m = 0;
  for (int k = 1; k <= nlev; ++k) {
    cd ck = 0.0;
    for (size_t q = 0; q < nd; ++q) ck += tv[q] * u[q];
    c[k - 1] = ck;
    for (size_t q = 0; q < nd; ++q) { re[q] = u[q].real(); im[q] = u[q].imag(); }
    augcls_apply(op, wk, re.data(), sre.data());
    augcls_apply(op, wk, im.data(), sim.data());
    augcls_rand_c(op, ep.data(), u.data(), dg.data());
    for (size_t q = 0; q < nd; ++q) w[q] = cd(sre[q], sim[q]) + dg[q];
    cd s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += u[q] * w[q];
    a[k - 1] = s;
    m = k;
    if (k == nlev) break;
    cd ak = a[k - 1], bk = k > 1 ? b[k - 2] : cd(0.0);
    for (size_t q = 0; q < nd; ++q) {
      w[q] = w[q] - ak * u[q];
      if (k > 1) w[q] = w[q] - bk * up[q];
    }
    if (project) augcls_project_c(op, w.data());
    s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += w[q] * w[q];
    b[k - 1] = std::sqrt(s);
    if (std::abs(b[k - 1]) < 1.0e-12) { closed = true; break; }
    bk = b[k - 1];
    for (size_t q = 0; q < nd; ++q) { up[q] = u[q]; u[q] = w[q] / bk; }
  }
  cf_species(a.data(), b.data(), c.data(), m, z, closed ? 0 : tail, g, f, nullptr, nullptr, nullptr);
}
extern "C" int orc_epi_blocks(void* h, int ns, const double* dc, const double* del, const double* enu, const double* v9,
                              double zr, double zi, int nlev, int tail, int project, double* x, int* mused) {
  Op& op = *(Op*)h;
  const cd z(zr, zi);
  size_t nd = 9 * (size_t)op.nn;
  std::vector<cd> ep(9 * (size_t)ns);
  for (int s = 0; s < ns; ++s)
    for (int l = 0; l < 9; ++l) ep[l + 9 * s] = z - dc[l] * (z - enu[l + 9 * s]) / del[l + 9 * s];
  std::vector<cd> s0(nd, 0.0), vv(nd, 0.0);
  for (int l = 0; l < 9; ++l) s0[l] = v9[l];
  hp_c(op, s0.data(), vv.data());
  if (project) augcls_project_c(op, vv.data());
  cd vn = 0.0;
  for (size_t q = 0; q < nd; ++q) vn += vv[q] * vv[q];
  double nv = std::sqrt(vn.real());
  if (nv < 1.0e-14) return fail("epi_start: zero start vector");
  cd g, fa, fb;
  int m0, m1;
  epi_chain(op, ep, s0, vv, z, nlev, tail, project != 0, g, fa, m0);
  cd* out = (cd*)x;
  out[0] = g;
  std::vector<cd> u1(nd);
  for (size_t q = 0; q < nd; ++q) u1[q] = vv[q] / nv;
  epi_chain(op, ep, u1, s0, z, nlev, tail, project != 0, g, fb, m1);
  out[2] = nv * nv * g;
  fb = nv * fb;
  out[1] = 0.5 * (fa + fb);
  out[3] = fa - fb;
  mused[0] = m0;
  mused[1] = m1;
  return 0;
}

// edc_green_proj src/asr_edc.f90:174-232: the chain of edc_green run all nlev steps (no depth test) with the projections
// of every Lanczos vector on the target states, cpr(k, l, t) = sum_ks tw(l, ks, t) psi_k(node ks of t, l), where psi is
// the unreduced amplitude augcls_amp_c (:251-261): csg(l, g) v(9 (r - 1) + pi(l, g)) / sq(r).  gp(l, t) =
// sum_k cpr(k, l, t) pv_k with pv from cf_species; gp4 the same with the chain cut four steps earlier.
// tnode, tgop (nsm, nt) 1-based (tnode 0: no node); tw (9, nsm, nt); gp, gp4 (9, nt) complex.
extern "C" void orc_edc_green_proj(void* h, int ns, const double* dc, const double* del, const double* enu, double zr,
                                   double zi, int iv, int nlev, int tail, int project, int nt, const int* tnode,
                                   const int* tgop, const double* tw, double* g, double* gp_out, double* gp4_out, int* mused) {
  Op& op = *(Op*)h;
  const int nsm = op.nsmax;
  const cd z(zr, zi);
  size_t nd = 9 * (size_t)op.nn;
  std::vector<cd> ep(9 * (size_t)ns);
  for (int s = 0; s < ns; ++s)
    for (int l = 0; l < 9; ++l) ep[l + 9 * s] = z - dc[l] * (z - enu[l + 9 * s]) / del[l + 9 * s];
  std::vector<cd> u(nd, 0.0), up(nd, 0.0), w(nd), dg(nd);
  std::vector<double> re(nd), im(nd), sre(nd), sim(nd);
  u[iv - 1] = 1.0;
  std::vector<cd> a(nlev, 0.0), b(nlev, 0.0), cc(nlev, 0.0), pv(nlev, 0.0);
  std::vector<cd> cpr((size_t)nlev * 9 * nt, 0.0);   // (k, l, t): k fastest
  int m = 0;
  Work wk;
  for (int k = 1; k <= nlev; ++k) {
    for (int t = 0; t < nt; ++t)
      for (int ks = 0; ks < nsm; ++ks) {
        int r = tnode[ks + (size_t)nsm * t];
        if (r <= 0) continue;
        int gg = tgop[ks + (size_t)nsm * t] - 1;
        for (int l = 0; l < 9; ++l) {
          cd amp = op.csg[l + 9 * gg] * u[9 * (size_t)(r - 1) + op.pi[l + 9 * gg] - 1] / op.sq[r - 1];
          cpr[(k - 1) + (size_t)nlev * (l + 9 * (size_t)t)] += tw[l + 9 * (ks + (size_t)nsm * t)] * amp;
        }
      }
    for (size_t q = 0; q < nd; ++q) { re[q] = u[q].real(); im[q] = u[q].imag(); }
    augcls_apply(op, wk, re.data(), sre.data());
    augcls_apply(op, wk, im.data(), sim.data());
    augcls_rand_c(op, ep.data(), u.data(), dg.data());
    for (size_t q = 0; q < nd; ++q) w[q] = cd(sre[q], sim[q]) + dg[q];
    cd s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += u[q] * w[q];
    a[k - 1] = s;
    m = k;
    if (k == nlev) break;
    cd ak = a[k - 1], bk = 0.0;
    if (k > 1) bk = b[k - 2];
    for (size_t q = 0; q < nd; ++q) {
      w[q] = w[q] - ak * u[q];
      if (k > 1) w[q] = w[q] - bk * up[q];
    }
    if (project) augcls_project_c(op, w.data());
    s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += w[q] * w[q];
    b[k - 1] = std::sqrt(s);
    if (std::abs(b[k - 1]) < 1.0e-12) break;
    bk = b[k - 1];
    for (size_t q = 0; q < nd; ++q) { up[q] = u[q]; u[q] = w[q] / bk; }
  }
  cd gg, ff;
  for (int pass = 0; pass < 2; ++pass) {
    int mm = pass == 0 ? m : std::max(1, m - 4);
    cf_species(a.data(), b.data(), cc.data(), mm, z, tail, gg, ff, nullptr, pv.data(), nullptr);
    if (pass == 0) { g[0] = gg.real(); g[1] = gg.imag(); }
    cd* out = (cd*)(pass == 0 ? gp_out : gp4_out);
    for (int t = 0; t < nt; ++t)
      for (int l = 0; l < 9; ++l) {
        cd acc = 0.0;
        for (int k = 0; k < mm; ++k) acc += cpr[k + (size_t)nlev * (l + 9 * (size_t)t)] * pv[k];
        out[l + 9 * (size_t)t] = acc;
      }
  }
  *mused = m;
}

// ---- block form: src/asr_augblk.f90 (rand_r :88-124, rand_lin_amp :127-165, smul :170-203, hmul :206-215,
//      blk_hamx :219-250, blk_project :284-304) and edc_green_blk src/asr_edc.f90:237-316.  Layout x(j, i): member fastest.
static bool uniform_par(const Op& op, const double* par) {
  for (int s = 1; s < op.nsp; ++s)
    for (int l = 0; l < 9; ++l) if (par[l + 9 * s] != par[l]) return false;
  return true;
}
static void rand_r(const Op& op, const double* par, const cd* x, cd* w, int nb) {
  const int nsm = op.nsmax;
  if (uniform_par(op, par)) {
    for (int i = 0; i < op.nn; ++i)
      for (int l = 0; l < 9; ++l)
        for (int j = 0; j < nb; ++j) { size_t q = j + nb * (9 * (size_t)i + l); w[q] = par[l] * x[q]; }
    return;
  }
  std::vector<double> wt;
  local_weights(op, par, wt);
  for (int i = 0; i < op.nn; ++i) {
    size_t j0 = 9 * (size_t)i;
    if (op.frozen[i] > 0) {
      for (int l = 0; l < 9; ++l)
        for (int j = 0; j < nb; ++j) w[j + nb * (j0 + l)] = par[l + 9 * (size_t)(op.frozen[i] - 1)] * x[j + nb * (j0 + l)];
      continue;
    }
    int kap = op.ncl[i] - 1, l0 = op.lst[i];
    for (int l = 0; l < 9; ++l)
      for (int j = 0; j < nb; ++j) w[j + nb * (j0 + l)] = WT(wt, l, l0, l0, kap) * x[j + nb * (j0 + l)];
    for (int k = 0; k < op.nsc[kap]; ++k) {
      int r = op.flipr[k + (size_t)nsm * i];
      if (k == l0 || r == 0) continue;
      int g = op.flipg[k + (size_t)nsm * i] - 1;
      size_t jr = 9 * (size_t)(r - 1);
      for (int l = 0; l < 9; ++l) {
        double f = WT(wt, l, l0, k, kap) * op.chi[g] * op.sg[l + 9 * g];
        for (int j = 0; j < nb; ++j) w[j + nb * (j0 + l)] = w[j + nb * (j0 + l)] + f * x[j + nb * (jr + op.pi[l + 9 * g] - 1)];
      }
    }
  }
}
static void rand_lin_amp(const Op& op, const double* pa, const double* pb, const cd* zs, const cd* x, cd* w, int nb) {
  const int nsm = op.nsmax;
  if (uniform_par(op, pa) && uniform_par(op, pb)) {
    for (int i = 0; i < op.nn; ++i)
      for (int l = 0; l < 9; ++l)
        for (int j = 0; j < nb; ++j) { size_t q = j + nb * (9 * (size_t)i + l); w[q] = (zs[j] * pa[l] + pb[l]) * x[q]; }
    return;
  }
  std::vector<double> wa, wb;
  local_weights(op, pa, wa); local_weights(op, pb, wb);
  for (int i = 0; i < op.nn; ++i) {
    size_t j0 = 9 * (size_t)i;
    if (op.frozen[i] > 0) {
      int s = op.frozen[i] - 1;
      for (int l = 0; l < 9; ++l)
        for (int j = 0; j < nb; ++j) w[j + nb * (j0 + l)] = (zs[j] * pa[l + 9 * s] + pb[l + 9 * s]) * x[j + nb * (j0 + l)];
      continue;
    }
    int kap = op.ncl[i] - 1, l0 = op.lst[i];
    for (int l = 0; l < 9; ++l)
      for (int j = 0; j < nb; ++j)
        w[j + nb * (j0 + l)] = (zs[j] * WT(wa, l, l0, l0, kap) + WT(wb, l, l0, l0, kap)) * x[j + nb * (j0 + l)];
    for (int k = 0; k < op.nsc[kap]; ++k) {
      int r = op.flipr[k + (size_t)nsm * i];
      if (k == l0 || r == 0) continue;
      int g = op.flipg[k + (size_t)nsm * i] - 1;
      size_t jr = 9 * (size_t)(r - 1);
      for (int l = 0; l < 9; ++l) {
        double fa = WT(wa, l, l0, k, kap) * op.chi[g] * op.sg[l + 9 * g];
        double fb = WT(wb, l, l0, k, kap) * op.chi[g] * op.sg[l + 9 * g];
        for (int j = 0; j < nb; ++j)
          w[j + nb * (j0 + l)] = w[j + nb * (j0 + l)] + (zs[j] * fa + fb) * x[j + nb * (jr + op.pi[l + 9 * g] - 1)];
      }
    }
  }
}
static void smul(const Op& op, const cd* t1, cd* t2, int nb) {
  const int ns = op.nslot, nop = op.nop;
  std::vector<cd> acc(9 * (size_t)nb);
  for (int i = 0; i < op.nn; ++i) {
    size_t j0 = 9 * (size_t)i;
    int t = op.stype[op.site[i] - 1] - 1;
    std::fill(acc.begin(), acc.end(), cd(0.0));
    for (int j = 0; j < nb; ++j)
      for (int l2 = 0; l2 < 9; ++l2) {
        cd s = t1[j + nb * (j0 + l2)];
        for (int l = 0; l < 9; ++l) acc[l + 9 * j] = acc[l + 9 * j] + op.block0[l + 9 * (l2 + 9 * (size_t)t)] * s;
      }
    for (int k = 0; k < ns; ++k) {
      int r = op.hopr[k + (size_t)ns * i];
      if (r == 0) continue;
      int g = op.hopg[k + (size_t)ns * i] - 1;
      size_t jr = 9 * (size_t)(r - 1);
      for (int l2 = 0; l2 < 9; ++l2) {
        double fc[9];
        const double* bt = &op.btab[9 * (l2 + 9 * (k + (size_t)ns * (g + (size_t)nop * t)))];
        for (int l = 0; l < 9; ++l) fc[l] = op.chi[g] * bt[l];
        for (int j = 0; j < nb; ++j) {
          cd v = t1[j + nb * (jr + l2)];
          for (int l = 0; l < 9; ++l) acc[l + 9 * j] = acc[l + 9 * j] + fc[l] * v;
        }
      }
    }
    for (int l = 0; l < 9; ++l)
      for (int j = 0; j < nb; ++j) t2[j + nb * (j0 + l)] = acc[l + 9 * j];
  }
}
static void hmul(const Op& op, const cd* x, cd* hx, cd* t1, cd* t2, int nb) {
  size_t nt = (size_t)nb * 9 * op.nn;
  rand_r(op, op.d.data(), x, t1, nb);
  smul(op, t1, t2, nb);
  rand_r(op, op.d.data(), t2, t1, nb);
  rand_r(op, op.c.data(), x, hx, nb);
  for (size_t q = 0; q < nt; ++q) hx[q] = hx[q] + t1[q];
}
struct BlkWork { int nb = 0; std::vector<cd> u, up, w, x0, h1, r1, h2, e1, t1, t2;
  void init(int nb_, size_t n) { nb = nb_; size_t m = (size_t)nb_ * n;
    for (auto* v : {&u, &up, &w, &x0, &h1, &r1, &h2, &e1, &t1, &t2}) v->assign(m, 0.0); } };
static void blk_hamx(const Op& op, BlkWork& wk, const double* pa, const double* pb, const cd* zs, const cd* x, cd* y) {
  const int nb = wk.nb;
  size_t nt = (size_t)nb * 9 * op.nn;
  for (int i = 0; i < op.nn; ++i)
    for (int l = 0; l < 9; ++l)
      for (int j = 0; j < nb; ++j) { size_t q = j + nb * (9 * (size_t)i + l); wk.x0[q] = x[q] / op.sq[i]; }
  hmul(op, wk.x0.data(), wk.h1.data(), wk.t1.data(), wk.t2.data(), nb);
  bool onz = false;
  for (double v : op.o) if (v != 0.0) onz = true;
  if (onz) {
    rand_r(op, op.o.data(), wk.h1.data(), wk.r1.data(), nb);
    hmul(op, wk.r1.data(), wk.h2.data(), wk.t1.data(), wk.t2.data(), nb);
    for (size_t q = 0; q < nt; ++q) wk.h1[q] = wk.h1[q] - wk.h2[q];
  }
  rand_lin_amp(op, pa, pb, zs, wk.x0.data(), wk.e1.data(), nb);
  bool enz = false;
  for (double v : op.e) if (v != 0.0) enz = true;
  if (enz) {
    rand_r(op, op.e.data(), wk.x0.data(), wk.r1.data(), nb);
    for (size_t q = 0; q < nt; ++q) wk.e1[q] = wk.e1[q] + wk.r1[q];
  }
  for (int i = 0; i < op.nn; ++i)
    for (int l = 0; l < 9; ++l)
      for (int j = 0; j < nb; ++j) { size_t q = j + nb * (9 * (size_t)i + l); y[q] = op.sq[i] * (wk.h1[q] + wk.e1[q]); }
}
static void blk_project(const Op& op, cd* x, int nb) {
  std::vector<cd> acc((size_t)nb * 9);
  for (int i = 0; i < op.nn; ++i) {
    int ns = op.stab_ptr[i + 1] - op.stab_ptr[i];
    if (ns <= 1) continue;
    size_t j0 = 9 * (size_t)i;
    std::fill(acc.begin(), acc.end(), cd(0.0));
    for (int jj = op.stab_ptr[i]; jj < op.stab_ptr[i + 1]; ++jj) {
      int g = op.stab[jj - 1] - 1;
      for (int l = 0; l < 9; ++l)
        for (int j = 0; j < nb; ++j)
          acc[j + (size_t)nb * l] = acc[j + (size_t)nb * l] + op.chi[g] * op.sg[l + 9 * g] * x[j + nb * (j0 + op.pi[l + 9 * g] - 1)];
    }
    for (int l = 0; l < 9; ++l)
      for (int j = 0; j < nb; ++j) x[j + nb * (j0 + l)] = acc[j + (size_t)nb * l] / (double)ns;
  }
}

// edc_green_blk src/asr_edc.f90:237-316.  zs(nb); outputs g(nb), mused(nb), a, b (nlev, nb) complex.
static void edc_green_blk(const Op& op, BlkWork& wk, const Edn& ed, const cd* zs, int nb, int iv, int nlev, double depth_tol,
                          int tail, bool project, cd* g, int* mused, cd* aout, cd* bout, long* nfall) {
  const int NB = wk.nb;
  std::vector<double> pa(9 * (size_t)ed.ns), pb(9 * (size_t)ed.ns);
  for (int s = 0; s < ed.ns; ++s)
    for (int l = 0; l < 9; ++l) {
      pa[l + 9 * s] = 1.0 - ed.dc[l] / ed.del[l + 9 * s];
      pb[l + 9 * s] = ed.dc[l] * ed.enu[l + 9 * s] / ed.del[l + 9 * s];
    }
  std::vector<cd> zp(NB);
  for (int j = 0; j < NB; ++j) zp[j] = zs[std::min(j, nb - 1)];
  size_t n = 9 * (size_t)op.nn;
  std::fill(wk.u.begin(), wk.u.end(), cd(0.0)); std::fill(wk.up.begin(), wk.up.end(), cd(0.0));
  for (int j = 0; j < nb; ++j) wk.u[j + (size_t)NB * (iv - 1)] = 1.0;
  std::vector<cd> a((size_t)nlev * NB, 0.0), b((size_t)nlev * NB, 0.0), cc(nlev, 0.0), gtry(NB), gprev(NB, 0.0), acc(NB);
  std::vector<int> m(NB, nlev);
  std::vector<char> act(NB, 0);
  std::vector<double> keep(NB);
  for (int j = 0; j < nb; ++j) act[j] = 1;
  cd ftmp;
  for (int k = 1; k <= nlev; ++k) {
    blk_hamx(op, wk, pa.data(), pb.data(), zp.data(), wk.u.data(), wk.w.data());
    std::fill(acc.begin(), acc.end(), cd(0.0));
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < NB; ++j) acc[j] = acc[j] + wk.u[j + NB * i] * wk.w[j + NB * i];
    for (int j = 0; j < NB; ++j) if (act[j]) { a[(k - 1) + (size_t)nlev * j] = acc[j]; m[j] = k; }
    if (k == nlev) break;
    if (depth_tol > 0.0 && k >= 8 && k % 4 == 0) {
      for (int j = 0; j < nb; ++j) {
        if (!act[j]) continue;
        cf_species(&a[(size_t)nlev * j], &b[(size_t)nlev * j], cc.data(), k, zs[j], tail, gtry[j], ftmp, nullptr, nullptr, nfall);
        if (k > 8 && std::abs(gtry[j] - gprev[j]) <= depth_tol * std::abs(gtry[j])) act[j] = 0;
        gprev[j] = gtry[j];
      }
    }
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < NB; ++j) {
        wk.w[j + NB * i] = wk.w[j + NB * i] - a[(k - 1) + (size_t)nlev * j] * wk.u[j + NB * i];
        if (k > 1) wk.w[j + NB * i] = wk.w[j + NB * i] - b[(k - 2) + (size_t)nlev * j] * wk.up[j + NB * i];
      }
    if (project) blk_project(op, wk.w.data(), NB);
    std::fill(acc.begin(), acc.end(), cd(0.0));
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < NB; ++j) acc[j] = acc[j] + wk.w[j + NB * i] * wk.w[j + NB * i];
    bool any = false;
    for (int j = 0; j < NB; ++j) {
      if (!act[j]) continue;
      b[(k - 1) + (size_t)nlev * j] = std::sqrt(acc[j]);
      if (std::abs(b[(k - 1) + (size_t)nlev * j]) < 1.0e-12) act[j] = 0;
    }
    for (int j = 0; j < NB; ++j) any = any || act[j];
    if (!any) break;
    for (int j = 0; j < NB; ++j) {
      if (act[j]) { acc[j] = 1.0 / b[(k - 1) + (size_t)nlev * j]; keep[j] = 1.0; }
      else { acc[j] = 0.0; keep[j] = 0.0; }
    }
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < NB; ++j) {
        wk.up[j + NB * i] = keep[j] * wk.u[j + NB * i];
        wk.u[j + NB * i] = acc[j] * wk.w[j + NB * i];
      }
  }
  for (int j = 0; j < nb; ++j) {
    cd fa;
    cf_species(&a[(size_t)nlev * j], &b[(size_t)nlev * j], cc.data(), m[j], zs[j], tail, g[j], fa, nullptr, nullptr, nfall);
    if (mused) mused[j] = m[j];
    if (aout) for (int k = 0; k < nlev; ++k) aout[k + (size_t)nlev * j] = a[k + (size_t)nlev * j];
    if (bout) for (int k = 0; k < nlev; ++k) bout[k + (size_t)nlev * j] = b[k + (size_t)nlev * j];
  }
}
extern "C" void orc_edc_green_blk(void* h, int ns, const double* dc, const double* del, const double* enu, const double* zs,
                                  int nb, int iv, int nlev, double depth_tol, int tail, int project, double* g, int* mused,
                                  double* a, double* b, long* nfall) {
  Op& op = *(Op*)h;
  Edn ed{ns, std::vector<double>(dc, dc + 9), std::vector<double>(del, del + 9 * ns), std::vector<double>(enu, enu + 9 * ns)};
  BlkWork wk;
  wk.init(nb, 9 * (size_t)op.nn);
  edc_green_blk(op, wk, ed, (const cd*)zs, nb, iv, nlev, depth_tol, tail, project != 0, (cd*)g, mused, (cd*)a, (cd*)b, nfall);
}

// ===================================================================================================== route ed3
// src/asr_ed3.f90: K'(z) = et - h' + u h' + h' u - h' Qt h' with h' = g + D_c^1/2 S D_c^1/2 (the operator's parameters
// c = g, d = D_c^1/2, o = e = 0 set by the caller, start site frozen to the central species); chains on z - K' from
// |a> = |u> + o_c |v> and |v> = h'|u>, each projected on the other start vector.
struct Ed3 { int ns; std::vector<double> dc, del, enu, o, p; };   // dc (9); del, enu, o, p (9, ns)

// ed3_coefs :91-107
static void ed3_coefs(const Ed3& ed, cd z, cd* et, cd* uu, cd* qt) {
  for (int s = 0; s < ed.ns; ++s)
    for (int l = 0; l < 9; ++l) {
      int q = l + 9 * s;
      cd eps = z - ed.enu[q];
      et[q] = ed.dc[l] / ed.del[q] * eps;
      uu[q] = ed.o[q] * eps;
      qt[q] = ed.del[q] / ed.dc[l] * (ed.o[q] - ed.p[q] * eps);
    }
}

// ed3_kmul :110-131: y = et x - h'x + u h'x + h'(u x - Qt h'x)
static void ed3_kmul(const Op& op, const cd* et, const cd* uu, const cd* qt, const cd* x, cd* y, std::vector<cd>* t) {
  size_t nd = 9 * (size_t)op.nn;
  hp_c(op, x, t[0].data());
  augcls_rand_c(op, qt, t[0].data(), t[1].data());
  augcls_rand_c(op, uu, x, t[2].data());
  for (size_t q = 0; q < nd; ++q) t[2][q] = t[2][q] - t[1][q];
  hp_c(op, t[2].data(), t[3].data());
  augcls_rand_c(op, et, x, y);
  augcls_rand_c(op, uu, t[0].data(), t[1].data());
  for (size_t q = 0; q < nd; ++q) y[q] = y[q] - t[0][q] + t[1][q] + t[3][q];
}

// cf_closed :221-236: the Krylov space is exhausted, the fraction is exact
static void cf_closed(const cd* a, const cd* b, const cd* c, int m, cd z, cd& g, cd& f) {
  std::vector<cd> gt(m);
  gt[m - 1] = 1.0 / (z - a[m - 1]);
  for (int j = m - 2; j >= 0; --j) gt[j] = 1.0 / (z - a[j] - b[j] * b[j] * gt[j + 1]);
  g = gt[0];
  f = 0.0;
  cd prod = gt[0];
  for (int k = 0; k < m; ++k) {
    f = f + c[k] * prod;
    if (k < m - 1) prod = prod * b[k] * gt[k + 1];
  }
}

// chain :147-218: one complex-symmetric chain on z - K' from start (start . start = 1), projections c_k = tv . u_k
static void ed3_chain(const Op& op, const cd* et, const cd* uu, const cd* qt, cd z, int nlev, double tnorm, double depth_tol,
                      int tail, bool project, const cd* start, const cd* tv, cd& g, cd& f, int& m, cd* acoef, cd* bcoef,
                      cd* ccoef, long* nfall) {
  size_t nd = 9 * (size_t)op.nn;
  std::vector<cd> u(start, start + nd), up(nd, 0.0), w(nd), t[4];
  for (auto& v : t) v.assign(nd, 0.0);
  std::vector<cd> a(nlev, 0.0), b(nlev, 0.0), c(nlev, 0.0);
  cd gprev = 0.0, fprev = 0.0, gtry, ftry;
  m = 0;
  bool closed = false;
  for (int k = 1; k <= nlev; ++k) {
    cd s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += tv[q] * u[q];
    c[k - 1] = s;
    ed3_kmul(op, et, uu, qt, u.data(), w.data(), t);
    for (size_t q = 0; q < nd; ++q) w[q] = z * u[q] - w[q];
    s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += u[q] * w[q];
    a[k - 1] = s;
    m = k;
    if (k == nlev) break;
    if (depth_tol > 0.0 && k >= 8 && k % 4 == 0) {
      cf_species(a.data(), b.data(), c.data(), k, z, tail, gtry, ftry, nullptr, nullptr, nfall);
      if (k > 8 && std::abs(gtry - gprev) <= depth_tol * std::abs(gtry) &&
          std::abs(ftry - fprev) <= depth_tol * std::max(std::abs(ftry), tnorm * std::abs(gtry)))
        break;
      gprev = gtry; fprev = ftry;
    }
    cd ak = a[k - 1], bk = 0.0;
    if (k > 1) bk = b[k - 2];
    for (size_t q = 0; q < nd; ++q) {
      w[q] = w[q] - ak * u[q];
      if (k > 1) w[q] = w[q] - bk * up[q];
    }
    if (project) augcls_project_c(op, w.data());
    s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += w[q] * w[q];
    b[k - 1] = std::sqrt(s);
    if (std::abs(b[k - 1]) < 1.0e-12) { closed = true; break; }
    bk = b[k - 1];
    for (size_t q = 0; q < nd; ++q) { up[q] = u[q]; u[q] = w[q] / bk; }
  }
  if (closed) cf_closed(a.data(), b.data(), c.data(), m, z, g, f);
  else cf_species(a.data(), b.data(), c.data(), m, z, tail, g, f, nullptr, nullptr, nfall);
  for (int k = 0; k < m; ++k) {
    if (acoef) acoef[k] = a[k];
    if (bcoef) bcoef[k] = b[k];
    if (ccoef) ccoef[k] = c[k];
  }
}

// ed3_start :135-144 and ed3_blocks :242-265 at one energy: bk(0) = G_11, bk(1) = (hG)_11, bk(2) = (hGh)_11,
// bk(3) = q1 of the |a> chain - q1 of the |v> chain.  m(2): depths of the two chains.
extern "C" int orc_ed3_blocks(void* h, int ns, const double* dc, const double* del, const double* enu, const double* o,
                              const double* p, int central, double zr, double zi, int iv, int nlev, double depth_tol, int tail,
                              int project, double* bk, int* mout, double* acoef, double* bcoef, double* ccoef, long* nfall) {
  Op& op = *(Op*)h;
  Ed3 ed{ns, std::vector<double>(dc, dc + 9), std::vector<double>(del, del + 9 * ns), std::vector<double>(enu, enu + 9 * ns),
         std::vector<double>(o, o + 9 * ns), std::vector<double>(p, p + 9 * ns)};
  size_t nd = 9 * (size_t)op.nn;
  std::vector<cd> s0(nd, 0.0), vv(nd), av(nd);
  s0[iv - 1] = 1.0;
  hp_c(op, s0.data(), vv.data());
  if (project) augcls_project_c(op, vv.data());
  const double oc = ed.o[(iv - 1) + 9 * (size_t)(central - 1)];
  for (size_t q = 0; q < nd; ++q) av[q] = s0[q] + oc * vv[q];
  cd sv = 0.0, sa = 0.0;
  for (size_t q = 0; q < nd; ++q) { sv += vv[q] * vv[q]; sa += av[q] * av[q]; }
  double nv = std::sqrt(sv.real()), na = std::sqrt(sa.real());
  if (nv < 1.0e-14 || na < 1.0e-14) return fail("ed3_start: zero start vector");
  cd z(zr, zi);
  std::vector<cd> et(9 * (size_t)ns), uu(9 * (size_t)ns), qt(9 * (size_t)ns);
  ed3_coefs(ed, z, et.data(), uu.data(), qt.data());
  std::vector<cd> st(nd);
  cd gt, fm;
  int m1 = 0, m2 = 0;
  for (size_t q = 0; q < nd; ++q) st[q] = av[q] / na;
  ed3_chain(op, et.data(), uu.data(), qt.data(), z, nlev, nv, depth_tol, tail, project != 0, st.data(), vv.data(), gt, fm, m1,
            acoef ? (cd*)acoef : nullptr, bcoef ? (cd*)bcoef : nullptr, ccoef ? (cd*)ccoef : nullptr, nfall);
  cd q0 = na * na * gt, q1a = na * fm;
  for (size_t q = 0; q < nd; ++q) st[q] = vv[q] / nv;
  ed3_chain(op, et.data(), uu.data(), qt.data(), z, nlev, na, depth_tol, tail, project != 0, st.data(), av.data(), gt, fm, m2,
            acoef ? (cd*)acoef + nlev : nullptr, bcoef ? (cd*)bcoef + nlev : nullptr, ccoef ? (cd*)ccoef + nlev : nullptr,
            nfall);
  cd q2 = nv * nv * gt, q1b = nv * fm;
  fm = 0.5 * (q1a + q1b);
  cd out[4] = {q0 - 2.0 * oc * fm + oc * oc * q2, fm - oc * q2, q2, q1a - q1b};
  for (int k = 0; k < 4; ++k) { bk[2 * k] = out[k].real(); bk[2 * k + 1] = out[k].imag(); }
  if (mout) { mout[0] = m1; mout[1] = m2; }
  return 0;
}

// ===================================================================================================== chain scheduler
// chain_greens / chain_worker src/asr_class_scf.f90:966-1160: tasks (energy block x start orbital x central species x
// spin), one block chain per task, dynamic schedule over the host threads.  Each task carries its own species parameters
// (the copy-on-write of lop(kp) = cop(kp)%op), its frozen start site and its start orbital.
// params: per (comp, spin) group q: c,d,o,e (9, nsp) each, then edn dc(9), del(9,nsp), enu(9,nsp); group layout
// [c|d|o|e|dc|del|enu] with sizes 4*9*nsp + 9 + 2*9*nsp.  gcomp(q): central species (frozen at the start site).
// iorb(o): start orbital index (1..9).  nlevq(q, o): chain depth.  Output gz(nz, norb, ngroup) complex; optional (NULL:
// not wanted) the chain coefficients a, b (ldab, nz, norb, ngroup) complex and the depths used mz(nz, norb, ngroup).
extern "C" int orc_chain_greens(void* h, int ngroup, const double* params, const int* gcomp, int norb, const int* iorb,
                                const int* nlevq, const double* zs, int nz, int nbe, double depth_tol, int tail, int project,
                                int nthreads, double* gz, long* nchainsteps, int ldab, double* az, double* bz, int* mz) {
  Op& op0 = *(Op*)h;
  const int nsp = op0.nsp;
  const size_t gstride = 4 * 9 * (size_t)nsp + 9 + 2 * 9 * (size_t)nsp;
  const int nbk = (nz + nbe - 1) / nbe;
  const long ntask = (long)nbk * norb * ngroup;
  long steps = 0;
  int err = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel reduction(+ : steps)
  {
    Op op = op0;   // per-thread copy: parameters, frozen and chi are private (src/asr_class_scf.f90:1110)
    BlkWork wk;
    wk.init(nbe, 9 * (size_t)op.nn);
    int curq = -1, curo = -1;
    std::vector<cd> gb(nbe), ab, bb;
    std::vector<int> mu(nbe);
#pragma omp for schedule(dynamic)
    for (long t = 0; t < ntask; ++t) {
      int jb = (int)(t % nbk), o = (int)((t / nbk) % norb), q = (int)(t / ((long)nbk * norb));
      const double* P = params + gstride * q;
      if (q != curq) {
        orc_set_params(&op, P, P + 9 * nsp, P + 18 * nsp, P + 27 * nsp);
        std::fill(op.frozen.begin(), op.frozen.end(), 0);
        if (gcomp[q] > 0 && orc_freeze_any(&op, 1, gcomp[q], nullptr)) { err = 1; }
        curq = q;
      }
      if (o != curo) { if (orc_set_start(&op, iorb[o])) err = 1; curo = o; }
      Edn ed{nsp, std::vector<double>(P + 36 * nsp, P + 36 * nsp + 9),
             std::vector<double>(P + 36 * nsp + 9, P + 36 * nsp + 9 + 9 * nsp),
             std::vector<double>(P + 36 * nsp + 9 + 9 * nsp, P + 36 * nsp + 9 + 18 * nsp)};
      int j1 = jb * nbe, j2 = std::min(nz, j1 + nbe);
      int nlev = nlevq[q + (size_t)ngroup * o];
      const bool want_ab = az && bz && nlev <= ldab;
      if (want_ab) { ab.assign((size_t)nlev * nbe, cd(0.0)); bb.assign((size_t)nlev * nbe, cd(0.0)); }
      edc_green_blk(op, wk, ed, (const cd*)zs + j1, j2 - j1, iorb[o], nlev, depth_tol, tail, project != 0, gb.data(), mu.data(),
                    want_ab ? ab.data() : nullptr, want_ab ? bb.data() : nullptr, nullptr);
      for (int j = j1; j < j2; ++j) {
        size_t dst = (size_t)j + (size_t)nz * (o + (size_t)norb * q);
        gz[2 * dst] = gb[j - j1].real(); gz[2 * dst + 1] = gb[j - j1].imag();
        steps += mu[j - j1];
        if (mz) mz[dst] = mu[j - j1];
        if (want_ab)
          for (int k = 0; k < nlev; ++k) {
            az[2 * (dst * ldab + k)] = ab[(size_t)(j - j1) * nlev + k].real();
            az[2 * (dst * ldab + k) + 1] = ab[(size_t)(j - j1) * nlev + k].imag();
            bz[2 * (dst * ldab + k)] = bb[(size_t)(j - j1) * nlev + k].real();
            bz[2 * (dst * ldab + k) + 1] = bb[(size_t)(j - j1) * nlev + k].imag();
          }
      }
    }
  }
  if (nchainsteps) *nchainsteps = steps;
  return err ? fail("orc_chain_greens: parameter setup failed") : 0;
}

// ===================================================================================================== contour
// src/asr_contour.f90:132-151 gauss_legendre
extern "C" void orc_gauss_legendre(int n, double* x, double* w) {
  for (int i = 1; i <= (n + 1) / 2; ++i) {
    double z = std::cos(PI * (i - 0.25) / (n + 0.5)), z1, p1, p2, p3, pp = 1.0;
    for (int it = 0; it < 100; ++it) {
      p1 = 1.0; p2 = 0.0;
      for (int k = 1; k <= n; ++k) { p3 = p2; p2 = p1; p1 = ((2 * k - 1) * z * p2 - (k - 1) * p3) / k; }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z; z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1.0e-15) break;
    }
    x[i - 1] = -z; x[n - i] = z;
    w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp); w[n - i] = w[i - 1];
  }
}
// contour_nodes :17-34 (eta_end < 0: absent)
extern "C" void orc_contour_nodes(double ebot, double ef, int n, double eta_end, double* z, double* w) {
  std::vector<double> x(n), wg(n);
  orc_gauss_legendre(n, x.data(), wg.data());
  double c = 0.5 * (ebot + ef), r = 0.5 * (ef - ebot), th0 = 0.0;
  if (eta_end >= 0.0) th0 = std::asin(std::min(eta_end / r, 0.5));
  for (int j = 0; j < n; ++j) {
    double th = th0 + 0.5 * (PI - th0) * (1.0 - x[j]);
    cd zz(c + r * std::cos(th), r * std::sin(th));
    cd ww = wg[j] * (-0.5 * (PI - th0)) * cd(0.0, r) * std::exp(cd(0.0, th));
    z[2 * j] = zz.real(); z[2 * j + 1] = zz.imag(); w[2 * j] = ww.real(); w[2 * j + 1] = ww.imag();
  }
}
// contour_nodes_closed :39-58
extern "C" void orc_contour_nodes_closed(double ebot, double ef, double eta, int na, int nv, double* z, double* w) {
  std::vector<double> xa(na), wa(na), xv(nv), wv(nv);
  orc_gauss_legendre(na, xa.data(), wa.data());
  orc_gauss_legendre(nv, xv.data(), wv.data());
  double c = (ef * ef + eta * eta - ebot * ebot) / (2.0 * (ef - ebot)), r = c - ebot, th0 = std::atan2(eta, ef - c);
  for (int j = 0; j < na; ++j) {
    double th = th0 + 0.5 * (PI - th0) * (1.0 - xa[j]);
    cd zz(c + r * std::cos(th), r * std::sin(th));
    cd ww = wa[j] * (-0.5 * (PI - th0)) * cd(0.0, r) * std::exp(cd(0.0, th));
    z[2 * j] = zz.real(); z[2 * j + 1] = zz.imag(); w[2 * j] = ww.real(); w[2 * j + 1] = ww.imag();
  }
  for (int j = 0; j < nv; ++j) {
    int k = na + j;
    z[2 * k] = ef; z[2 * k + 1] = 0.5 * eta * (1.0 + xv[j]);
    w[2 * k] = 0.0; w[2 * k + 1] = -0.5 * eta * wv[j];
  }
}
// contour_nodes_fermi :77-121 (Wildberger et al., PRB 52, 11502 (1995))
extern "C" void orc_contour_nodes_fermi(double ebot, double mu, double kt, int npole, int nmain, int nstep, double* z, double* w) {
  auto fermi_r = [&](double e) { double t = (e - mu) / kt; return t > 0.0 ? std::exp(-t) / (1.0 + std::exp(-t)) : 1.0 / (1.0 + std::exp(t)); };
  auto fermi_c = [&](cd zz) { cd t = (zz - mu) / kt; return t.real() < -600.0 ? cd(1.0) : 1.0 / (std::exp(t) + 1.0); };
  double gam = 2.0 * npole * PI * kt;
  std::vector<double> xv(4), wv(4), xm(nmain), wm(nmain), xs(nstep), ws(nstep), xt(8), wt(8);
  orc_gauss_legendre(4, xv.data(), wv.data()); orc_gauss_legendre(nmain, xm.data(), wm.data());
  orc_gauss_legendre(nstep, xs.data(), ws.data()); orc_gauss_legendre(8, xt.data(), wt.data());
  int k = 0;
  auto put = [&](cd zz, cd ww) { z[2 * k] = zz.real(); z[2 * k + 1] = zz.imag(); w[2 * k] = ww.real(); w[2 * k + 1] = ww.imag(); ++k; };
  for (int j = 0; j < 4; ++j) { cd zz(ebot, 0.5 * gam * (1.0 + xv[j])); put(zz, cd(0.0, 0.5 * gam * wv[j]) * fermi_c(zz)); }
  double lo = ebot, hi = mu - 10.0 * kt;
  for (int j = 0; j < nmain; ++j) { double x = 0.5 * (lo + hi) + 0.5 * (hi - lo) * xm[j]; put(cd(x, gam), 0.5 * (hi - lo) * wm[j] * fermi_r(x)); }
  lo = mu - 10.0 * kt; hi = mu + 10.0 * kt;
  for (int j = 0; j < nstep; ++j) { double x = 0.5 * (lo + hi) + 0.5 * (hi - lo) * xs[j]; put(cd(x, gam), 0.5 * (hi - lo) * ws[j] * fermi_r(x)); }
  lo = mu + 10.0 * kt; hi = mu + 40.0 * kt;
  for (int j = 0; j < 8; ++j) { double x = 0.5 * (lo + hi) + 0.5 * (hi - lo) * xt[j]; put(cd(x, gam), 0.5 * (hi - lo) * wt[j] * fermi_r(x)); }
  for (int j = 0; j < npole; ++j) put(cd(mu, (2 * j + 1) * PI * kt), cd(0.0, -2.0 * PI * kt));
}
// contour_moment :124-130
extern "C" double orc_contour_moment(const double* z, const double* w, const double* g, int n, double enu, int k) {
  cd s = 0.0;
  for (int j = 0; j < n; ++j) s += cd(w[2 * j], w[2 * j + 1]) * std::pow(cd(z[2 * j], z[2 * j + 1]) - enu, k) * cd(g[2 * j], g[2 * j + 1]);
  return -s.imag() / PI;
}

// ===================================================================================================== KPM
// kpm_moments / kpm_dos src/reference/asr_kpm.f90:39-87 on an explicit supercell operator (lmto_real_op,
// src/reference/asr_lmto_realization.f90:120-191, generalised to n species; o = 0 gives H = E + h).
// Rademacher vectors come from the counter-based generator below (the Fortran RNG is compiler-specific): entry q of
// vector v is +1 if bit 63 of splitmix64(seed * 0x9E3779B97F4A7C15 + (v << 40) + q) is clear, else -1.  The GPU kernels use
// the same definition, so FP64 parity is exact in law and in value.
static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
extern "C" double orc_rademacher(uint64_t seed, uint64_t v, uint64_t q) {
  return (splitmix64(seed * 0x9E3779B97F4A7C15ULL + (v << 40) + q) >> 63) ? -1.0 : 1.0;
}
struct RealOp {  // nsite sites, nslot neighbour slots, per-site species
  int n, ns;
  const int* nbr;        // (ns, n) 1-based
  const int* spc;        // (n) species 1..nsp
  const double *c, *d, *o, *e;   // (9, nsp)
  const double* block;   // (9, 9, ns)
  const double* block0;  // (9, 9)
};
static void real_h_apply(const RealOp& R, const double* x, double* hx, std::vector<double>& t) {   // h_apply :120-147
  size_t nd = 9 * (size_t)R.n;
  t.resize(nd);
  for (int i = 0; i < R.n; ++i) {
    int s = R.spc[i] - 1;
    for (int l = 0; l < 9; ++l) t[9 * (size_t)i + l] = R.d[l + 9 * s] * x[9 * (size_t)i + l];
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < R.n; ++i) {
    int s = R.spc[i] - 1;
    for (int l = 0; l < 9; ++l) {
      double acc = 0.0;
      for (int l2 = 0; l2 < 9; ++l2) acc = acc + R.block0[l + 9 * l2] * t[9 * (size_t)i + l2];
      for (int k = 0; k < R.ns; ++k) {
        int j = R.nbr[k + (size_t)R.ns * i] - 1;
        for (int l2 = 0; l2 < 9; ++l2) acc = acc + R.block[l + 9 * (l2 + 9 * (size_t)k)] * t[9 * (size_t)j + l2];
      }
      hx[9 * (size_t)i + l] = R.c[l + 9 * s] * x[9 * (size_t)i + l] + R.d[l + 9 * s] * acc;
    }
  }
}
static void real_apply(const RealOp& R, const double* x, double* y) {   // real_apply :149-191 (order 2)
  size_t nd = 9 * (size_t)R.n;
  std::vector<double> hx(nd), w(nd), hw(nd), t;
  real_h_apply(R, x, hx.data(), t);
  bool onz = false;
  for (int i = 0; i < R.n && !onz; ++i) for (int l = 0; l < 9; ++l) if (R.o[l + 9 * (R.spc[i] - 1)] != 0.0) onz = true;
  if (onz) {
    for (int i = 0; i < R.n; ++i) for (int l = 0; l < 9; ++l) w[9 * (size_t)i + l] = R.o[l + 9 * (R.spc[i] - 1)] * hx[9 * (size_t)i + l];
    real_h_apply(R, w.data(), hw.data(), t);
  }
  for (int i = 0; i < R.n; ++i)
    for (int l = 0; l < 9; ++l) {
      size_t q = 9 * (size_t)i + l;
      y[q] = R.e[l + 9 * (R.spc[i] - 1)] * x[q] + hx[q] - (onz ? hw[q] : 0.0);
    }
}
extern "C" void orc_real_apply(int n, int ns, const int* nbr, const int* spc, const double* c, const double* d, const double* o,
                               const double* e, const double* block, const double* block0, const double* x, double* y) {
  RealOp R{n, ns, nbr, spc, c, d, o, e, block, block0};
  real_apply(R, x, y);
}
// mu(0:nmom-1) averaged over vectors v0 .. v0+nvec-1 (the caller may split the vectors)
extern "C" void orc_kpm_moments(int n, int ns, const int* nbr, const int* spc, const double* c, const double* d, const double* o,
                                const double* e, const double* block, const double* block0, double cen, double sc, int nmom,
                                int v0, int nvec, uint64_t seed, double* mu) {
  RealOp R{n, ns, nbr, spc, c, d, o, e, block, block0};
  size_t nd = 9 * (size_t)n;
  std::vector<double> r(nd), t0(nd), t1(nd), t2(nd), w(nd);
  for (int k = 0; k < nmom; ++k) mu[k] = 0.0;
  for (int iv = v0; iv < v0 + nvec; ++iv) {
    for (size_t q = 0; q < nd; ++q) r[q] = orc_rademacher(seed, iv, q);
    t0 = r;
    real_apply(R, r.data(), w.data());
    for (size_t q = 0; q < nd; ++q) t1[q] = (w[q] - cen * r[q]) / sc;
    double s = 0.0;
    for (size_t q = 0; q < nd; ++q) s += r[q] * t0[q];
    mu[0] += s / (double)nd;
    if (nmom > 1) { s = 0.0; for (size_t q = 0; q < nd; ++q) s += r[q] * t1[q]; mu[1] += s / (double)nd; }
    for (int m = 2; m < nmom; ++m) {
      real_apply(R, t1.data(), w.data());
      for (size_t q = 0; q < nd; ++q) t2[q] = 2.0 * (w[q] - cen * t1[q]) / sc - t0[q];
      s = 0.0;
      for (size_t q = 0; q < nd; ++q) s += r[q] * t2[q];
      mu[m] += s / (double)nd;
      std::swap(t0, t1); std::swap(t1, t2);
    }
  }
  for (int k = 0; k < nmom; ++k) mu[k] /= (double)nvec;
}
// kpm_dos :68-87 (Jackson kernel)
extern "C" void orc_kpm_dos(const double* mu, int nmom, double cen, double sc, const double* e, int ne, double* rho) {
  std::vector<double> g(nmom);
  for (int n = 0; n < nmom; ++n)
    g[n] = ((nmom - n + 1) * std::cos(PI * n / (nmom + 1)) + std::sin(PI * n / (nmom + 1)) / std::tan(PI / (nmom + 1))) / (nmom + 1);
  for (int i = 0; i < ne; ++i) {
    double x = (e[i] - cen) / sc;
    if (std::fabs(x) >= 1.0) { rho[i] = 0.0; continue; }
    double th = std::acos(x), s = g[0] * mu[0];
    for (int n = 1; n < nmom; ++n) s = s + 2.0 * g[n] * mu[n] * std::cos(n * th);
    rho[i] = s / (PI * std::sqrt(1.0 - x * x) * sc);
  }
}
