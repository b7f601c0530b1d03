// Device construction of the augmented-space node set and its index maps: build_augcls_operator
// (src/asr_augcls.f90:596-823) with canon_node (:494-526), set_state / get_state (:207-235).
//
// The reference inserts candidates serially in the order (node, k1, k2, f) of its breadth-first loop, so a node's index
// is the position of the first candidate that produced it.  Here every level is expanded in parallel:
//   1. one thread per (node, k1, k2) triple counts its candidates; an exclusive scan gives each candidate its position
//      in the serial order;
//   2. one thread per triple writes its candidates' canonical keys (site, sorted configuration codes padded with
//      INT_MAX) at those positions;
//   3. one thread per candidate claims its key in an open-addressing table: existing nodes are found as node ids, new
//      keys are claimed by the smallest candidate position (atomicMax on the encoded position);
//   4. the first candidate of every new key gets index n_old + (number of first candidates before it), found by a
//      second scan, and writes the node record.
// The result is the reference's numbering for any thread count.  Levels are processed in node chunks bounded in
// candidate count; the order across chunks is the serial order, so chunking does not change the numbering.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <string>
#include <type_traits>
#include <vector>

#include "op.h"

namespace asrb {
namespace {

constexpr int RMAX = 15;            // configuration codes per key
constexpr int EMPTY = -1;
constexpr signed char CAND_SKIP = 0, CAND_VALID = 1, CAND_EXIST = 2;

struct BuildView {
  int n, nop, nsm, W, R, rkmax, maxdeg;
  const int* nbr_ptr;   // (n+1) 1-based
  const int* nbr;       // 1-based
  const int* perm;      // (n, nop)
  const int* nst;       // (n) allowed local states
};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
  return x;
}
__device__ __forceinline__ uint32_t key_hash(const int* k, int W) {
  uint64_t h = 0x9E3779B97F4A7C15ULL;
  for (int q = 0; q < W; ++q) h = mix64(h ^ (uint64_t)(uint32_t)k[q] * 0x100000001B3ULL + (uint64_t)q);
  return (uint32_t)(h >> 17);
}
__device__ __forceinline__ bool key_eq(const int* a, const int* b, int W) {
  for (int q = 0; q < W; ++q) if (a[q] != b[q]) return false;
  return true;
}
__device__ __forceinline__ void sort_small(int* a, int n) {
  for (int i = 1; i < n; ++i) {
    int t = a[i], j = i - 1;
    while (j >= 0 && a[j] > t) { a[j + 1] = a[j]; --j; }
    a[j + 1] = t;
  }
}
// set_state (src/asr_augcls.f90:217-235) in place: remove site r, then insert r*nsm + k (k > 0) in sorted position
__device__ __forceinline__ int set_state(int* cfg, int n, int r, int k, int nsm) {
  int m = 0;
  for (int i = 0; i < n; ++i) if (cfg[i] / nsm != r) cfg[m++] = cfg[i];
  if (k > 0) {
    int code = r * nsm + k, i = m;
    cfg[m++] = code;
    while (i > 0 && cfg[i - 1] > cfg[i]) { int t = cfg[i]; cfg[i] = cfg[i - 1]; cfg[i - 1] = t; --i; }
  }
  return m;
}
// canon_node (src/asr_augcls.f90:494-526): lexicographic minimum of (site, sorted codes) over the operations
__device__ void canon_node(const BuildView& B, int s, const int* cfg, int n, int* ccfg, int& csite, int& osize, int& gbest) {
  int c2[RMAX];
  csite = INT_MAX;
  for (int k = 0; k < n; ++k) ccfg[k] = INT_MAX;
  int ntie = 0;
  gbest = 0;
  for (int iop = 0; iop < B.nop; ++iop) {
    const int* p = B.perm + (size_t)iop * B.n;
    int s2 = p[s - 1];
    for (int k = 0; k < n; ++k) c2[k] = p[cfg[k] / B.nsm - 1] * B.nsm + cfg[k] % B.nsm;
    sort_small(c2, n);
    bool better = false, equal = false;
    if (s2 < csite) better = true;
    else if (s2 == csite) {
      equal = true;
      for (int k = 0; k < n; ++k) {
        if (c2[k] < ccfg[k]) { better = true; equal = false; break; }
        if (c2[k] > ccfg[k]) { equal = false; break; }
      }
    }
    if (better) { csite = s2; for (int k = 0; k < n; ++k) ccfg[k] = c2[k]; ntie = 1; gbest = iop; }
    else if (equal) ++ntie;
  }
  osize = B.nop / ntie;
}
__device__ __forceinline__ int key_len(const int* key, int W) {
  int n = 0;
  for (int q = 1; q < W; ++q) if (key[q] != INT_MAX) ++n;
  return n;
}
__device__ __forceinline__ int nbr_of(const BuildView& B, int r, int k) {   // k = 0: the site itself
  return k == 0 ? r : B.nbr[B.nbr_ptr[r - 1] - 1 + k - 1];
}
__device__ __forceinline__ int deg_of(const BuildView& B, int r) { return B.nbr_ptr[r] - B.nbr_ptr[r - 1]; }

// triple t of node chunk [a, b): node a + t / T2, k1 = (t / T1) % T1, k2 = t % T1, T1 = maxdeg + 1
__device__ bool triple_sites(const BuildView& B, const int* keys, int node, int k1, int k2, int* sites, int& nsit, int* err) {
  int r = keys[(size_t)node * B.W];
  if (k1 > deg_of(B, r)) return false;
  int r1 = nbr_of(B, r, k1);
  if (r1 == 0) return false;
  if (r1 < 0) { dev_fail(err, DERR_EDGE); return false; }
  if (k2 > deg_of(B, r1)) return false;
  int r2 = nbr_of(B, r1, k2);
  if (r2 == 0) return false;
  if (r2 < 0) { dev_fail(err, DERR_EDGE); return false; }
  nsit = 1; sites[0] = r;
  if (r1 != r) sites[nsit++] = r1;
  if (r2 != r && r2 != r1) sites[nsit++] = r2;
  sites[3] = r2;
  return true;
}

__global__ void k_count(BuildView B, const int* keys, int a, int ntrip, int* cnt, int* err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntrip) return;
  const int T1 = B.maxdeg + 1, T2 = T1 * T1;
  int node = a + t / T2, k1 = (t / T1) % T1, k2 = t % T1;
  int sites[4], nsit;
  int c = 0;
  if (triple_sites(B, keys, node, k1, k2, sites, nsit, err)) {
    c = 1;
    for (int j = 0; j < nsit; ++j) c *= B.nst[sites[j] - 1];
  }
  cnt[t] = c;
}

__global__ void k_generate(BuildView B, const int* keys, int a, int ntrip, const int* off, int* ckey, int* cosz,
                           signed char* cstat, int* err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntrip) return;
  const int T1 = B.maxdeg + 1, T2 = T1 * T1;
  int node = a + t / T2, k1 = (t / T1) % T1, k2 = t % T1;
  int sites[4], nsit;
  if (!triple_sites(B, keys, node, k1, k2, sites, nsit, err)) return;
  const int* nk = keys + (size_t)node * B.W;
  int n0 = key_len(nk, B.W);
  int ncomb = 1;
  for (int j = 0; j < nsit; ++j) ncomb *= B.nst[sites[j] - 1];
  int base = off[t];
  int cc[RMAX + 3], ccf[RMAX];
  for (int f = 0; f < ncomb; ++f) {
    int n = n0;
    for (int q = 0; q < n0; ++q) cc[q] = nk[1 + q];
    int q = f;
    for (int j = 0; j < nsit; ++j) {
      int ns_ = B.nst[sites[j] - 1];
      if (ns_ == 1) continue;
      int dgt = q % ns_;
      q /= ns_;
      n = set_state(cc, n, sites[j], dgt, B.nsm);
    }
    int* out = ckey + (size_t)(base + f) * B.W;
    if (n > B.rkmax) { cstat[base + f] = CAND_SKIP; continue; }
    if (n > B.R) { dev_fail(err, DERR_KEY); cstat[base + f] = CAND_SKIP; continue; }
    int cs, osz, gb;
    canon_node(B, sites[3], cc, n, ccf, cs, osz, gb);
    out[0] = cs;
    for (int k = 0; k < B.R; ++k) out[1 + k] = k < n ? ccf[k] : INT_MAX;
    cosz[base + f] = osz;
    cstat[base + f] = CAND_VALID;
  }
}

__global__ void k_insert(int C, int W, const int* ckey, signed char* cstat, const int* nkey, int* table, uint32_t tmask,
                         int* err) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C || cstat[c] != CAND_VALID) return;
  const int* key = ckey + (size_t)c * W;
  uint32_t h = key_hash(key, W) & tmask;
  const int enc = -c - 2;
  for (uint32_t p = 0; p <= tmask; ++p) {
    int v = atomicAdd(&table[h], 0);
    if (v == EMPTY) {
      int prev = atomicCAS(&table[h], EMPTY, enc);
      if (prev == EMPTY) return;
      v = prev;
    }
    if (v >= 0) {
      if (key_eq(nkey + (size_t)v * W, key, W)) { cstat[c] = CAND_EXIST; return; }
    } else {
      if (key_eq(ckey + (size_t)(-v - 2) * W, key, W)) { atomicMax(&table[h], enc); return; }
    }
    h = (h + 1) & tmask;
  }
  dev_fail(err, DERR_TABLE_FULL);
}

__global__ void k_first(int C, int W, const int* ckey, const signed char* cstat, const int* table, uint32_t tmask,
                        int* first, int* slot, int* err) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  first[c] = 0;
  if (cstat[c] != CAND_VALID) return;
  const int* key = ckey + (size_t)c * W;
  uint32_t h = key_hash(key, W) & tmask;
  for (uint32_t p = 0; p <= tmask; ++p) {
    int v = table[h];
    if (v <= -2 && key_eq(ckey + (size_t)(-v - 2) * W, key, W)) {
      first[c] = (v == -c - 2) ? 1 : 0;
      slot[c] = (int)h;
      return;
    }
    if (v == EMPTY) break;
    h = (h + 1) & tmask;
  }
  dev_fail(err, DERR_TABLE_FULL);
}

__global__ void k_commit(int C, int W, const int* ckey, const int* cosz, const int* first, const int* pos, const int* slot,
                         int nbase, int lev, int* nkey, int* nlevel, int* norb, int* table) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C || !first[c]) return;
  int id = nbase + pos[c];
  for (int q = 0; q < W; ++q) nkey[(size_t)id * W + q] = ckey[(size_t)c * W + q];
  nlevel[id] = lev;
  norb[id] = cosz[c];
  table[slot[c]] = id;
}

__global__ void k_rehash(int nn, int W, const int* nkey, int* table, uint32_t tmask, int* err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  uint32_t h = key_hash(nkey + (size_t)i * W, W) & tmask;
  for (uint32_t p = 0; p <= tmask; ++p) {
    if (atomicCAS(&table[h], EMPTY, i) == EMPTY) return;
    h = (h + 1) & tmask;
  }
  dev_fail(err, DERR_TABLE_FULL);
}

__device__ int find_node(int W, const int* key, const int* nkey, const int* table, uint32_t tmask) {
  uint32_t h = key_hash(key, W) & tmask;
  for (uint32_t p = 0; p <= tmask; ++p) {
    int v = table[h];
    if (v == EMPTY) return -1;
    if (v >= 0 && key_eq(nkey + (size_t)v * W, key, W)) return v;
    h = (h + 1) & tmask;
  }
  return -1;
}

// stabiliser {g : g site = site, g cfg = cfg}
__device__ int stab_ops(const BuildView& B, const int* nk, uint8_t* out) {
  int r = nk[0];
  int n = key_len(nk, B.W);
  int c2[RMAX];
  int cnt = 0;
  for (int g = 0; g < B.nop; ++g) {
    const int* p = B.perm + (size_t)g * B.n;
    if (p[r - 1] != r) continue;
    for (int k = 0; k < n; ++k) c2[k] = p[nk[1 + k] / B.nsm - 1] * B.nsm + nk[1 + k] % B.nsm;
    sort_small(c2, n);
    bool eq = true;
    for (int k = 0; k < n; ++k) if (c2[k] != nk[1 + k]) { eq = false; break; }
    if (eq) { if (out) out[cnt] = (uint8_t)g; ++cnt; }
  }
  return cnt;
}

__global__ void k_stab_count(BuildView B, int nn, const int* nkey, const int* norb, int* cnt, int* err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  int c = stab_ops(B, nkey + (size_t)i * B.W, nullptr);
  if (c * norb[i] != B.nop) dev_fail(err, DERR_STAB);
  cnt[i] = c;
}

struct TableOut {
  int* site; int8_t* lst; int8_t* ncl; int8_t* typ; int8_t* start; double* sq; double* isq;
  int* flipr; uint8_t* flipg; int* hopr; uint8_t* hopg; const int* stab_ptr; uint8_t* stab;
};

__global__ void k_tables(BuildView B, int nn, int nslot, const int* nkey, const int* norb, const int* table, uint32_t tmask,
                         const int* cls, const int* nsc, const int* canflip, const int* stype, int start_site, TableOut T) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const int* nk = nkey + (size_t)i * B.W;
  int r = nk[0];
  int n0 = key_len(nk, B.W);
  stab_ops(B, nk, T.stab + T.stab_ptr[i]);
  double no = (double)norb[i];
  T.sq[i] = sqrt(no);
  T.isq[i] = 1.0 / sqrt(no);
  T.site[i] = r;
  int kap = cls[r - 1];
  T.ncl[i] = (int8_t)(kap - 1);
  T.typ[i] = (int8_t)(stype[r - 1] - 1);
  T.start[i] = (int8_t)(r == start_site);
  int lst = 0;   // get_state (src/asr_augcls.f90:208-215)
  for (int q = 0; q < n0; ++q) if (nk[1 + q] / B.nsm == r) { lst = nk[1 + q] % B.nsm; break; }
  T.lst[i] = (int8_t)lst;
  int cc[RMAX + 1], ccf[RMAX], key[RMAX + 1];
  for (int k = 0; k < B.nsm; ++k) { T.flipr[k + (size_t)B.nsm * i] = -1; T.flipg[k + (size_t)B.nsm * i] = 0; }
  for (int k = 0; k < nsc[kap - 1]; ++k) {
    if (k == lst) { T.flipr[k + (size_t)B.nsm * i] = i; T.flipg[k + (size_t)B.nsm * i] = 0; continue; }
    if (!(k == 0 || canflip[r - 1])) continue;
    for (int q = 0; q < n0; ++q) cc[q] = nk[1 + q];
    int n = set_state(cc, n0, r, k, B.nsm);
    if (n > B.R) continue;   // longer than any stored node: not in the node set
    int cs, osz, gb;
    canon_node(B, r, cc, n, ccf, cs, osz, gb);
    key[0] = cs;
    for (int q = 0; q < B.R; ++q) key[1 + q] = q < n ? ccf[q] : INT_MAX;
    int j = find_node(B.W, key, nkey, table, tmask);
    if (j >= 0) { T.flipr[k + (size_t)B.nsm * i] = j; T.flipg[k + (size_t)B.nsm * i] = (uint8_t)gb; }
  }
  int deg = deg_of(B, r);
  for (int k = 0; k < nslot; ++k) { T.hopr[k + (size_t)nslot * i] = -1; T.hopg[k + (size_t)nslot * i] = 0; }
  for (int k = 0; k < deg; ++k) {
    int nb = B.nbr[B.nbr_ptr[r - 1] - 1 + k];
    if (nb <= 0) continue;
    int cs, osz, gb;
    canon_node(B, nb, nk + 1, n0, ccf, cs, osz, gb);
    key[0] = cs;
    for (int q = 0; q < B.R; ++q) key[1 + q] = q < n0 ? ccf[q] : INT_MAX;
    int j = find_node(B.W, key, nkey, table, tmask);
    if (j >= 0) { T.hopr[k + (size_t)nslot * i] = j; T.hopg[k + (size_t)nslot * i] = (uint8_t)gb; }
  }
}

// target links (src/asr_augcls.f90:808-820): for target t and local state k, the site alone in state k (every other site
// in its reference state) canonicalised and looked up; tnode 1-based (0: not in the node set), tgop 1-based operation
__global__ void k_targets(BuildView B, int nt, const int* tsite, const int* nkey, const int* table, uint32_t tmask,
                          const int* cls, const int* nsc, const int* canflip, int start_site, int* tnode, int* tgop) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nt * B.nsm) return;
  int t = q / B.nsm, k = q % B.nsm;
  int r = tsite[t];
  tnode[q] = 0;
  tgop[q] = 1;
  if (k >= nsc[cls[r - 1] - 1]) return;
  if (k > 0 && (r == start_site || !canflip[r - 1])) return;
  int cc[RMAX + 1], ccf[RMAX], key[RMAX + 1];
  int n = 0;
  if (k > 0) cc[n++] = r * B.nsm + k;
  if (n > B.R) return;
  int cs, osz, gb;
  canon_node(B, r, cc, n, ccf, cs, osz, gb);
  key[0] = cs;
  for (int p = 0; p < B.R; ++p) key[1 + p] = p < n ? ccf[p] : INT_MAX;
  int j = find_node(B.W, key, nkey, table, tmask);
  tgop[q] = gb + 1;
  if (j >= 0) tnode[q] = j + 1;
}

// ---------------------------------------------------------------------------------------------------- host side
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DBuf() { if (p) cudaFree(p); }
  int alloc(size_t m) {
    if (m <= n && p) return ASR_OK;
    if (p) cudaFree(p);
    p = nullptr; n = 0;
    if (cudaMalloc(&p, std::max<size_t>(m, 1) * sizeof(T)) != cudaSuccess) {
      set_error("graph build: device allocation of %zu bytes failed", m * sizeof(T));
      return ASR_ENOMEM;
    }
    n = m;
    return ASR_OK;
  }
  int grow_keep(size_t m, cudaStream_t s) {   // grow, keeping contents
    if (m <= n && p) return ASR_OK;
    size_t nm = std::max(m, 2 * n);
    T* q = nullptr;
    if (cudaMalloc(&q, nm * sizeof(T)) != cudaSuccess) {
      set_error("graph build: device allocation of %zu bytes failed", nm * sizeof(T));
      return ASR_ENOMEM;
    }
    if (p) { cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, s); cudaStreamSynchronize(s); cudaFree(p); }
    p = q; n = nm;
    return ASR_OK;
  }
  T* release() { T* q = p; p = nullptr; n = 0; return q; }
};

int check_err(asr_ctx* ctx, const char* where) {
  int h = 0;
  ASR_CUDA(cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  ASR_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h == DERR_NONE) return ASR_OK;
  cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream);
  switch (h) {
    case DERR_EDGE: set_error("build_augcls_operator: the closure reaches the edge of the site cluster (%s)", where); return ASR_EEDGE;
    case DERR_STAB: set_error("build_augcls_operator: stabiliser size /= group order / orbit size (%s)", where); return ASR_ESTATE;
    case DERR_KEY: set_error("build_augcls_operator: configuration longer than the key width (%s)", where); return ASR_ESTATE;
    default: set_error("build_augcls_operator: node hash table overflow (%s)", where); return ASR_ESTATE;
  }
}

template <typename T>
int exclusive_scan(const T* in, T* out, int n, DBuf<unsigned char>& tmp, cudaStream_t s) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s);
  ASR_TRY(tmp.alloc(bytes));
  ASR_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, n, s));
  return ASR_OK;
}

inline int blocks(long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

// ---------------------------------------------------------------------------------------------------- node order
// The build numbers nodes in the reference's serial order (breadth-first over two-hop candidates), in which the hop
// neighbours of a node lie a median of ~1e3 nodes away (up to the width of a level).  The chain kernels gather the 9
// orbital rows of every hop neighbour, so the device keeps its tables in a reverse Cuthill-McKee order of the hop graph
// (start node kept first), where the neighbours lie within ~1e2 nodes and the gathers stay in L2.  Results do not
// depend on the order: every vector and table is permuted consistently, and the host interfaces translate.
template <typename T>
__global__ void k_perm_rows(int nn, int w, const int* old_of_new, const int* new_of_old, const T* in, T* out, bool remap) {
  long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)nn * w) return;
  int n = (int)(q / w), k = (int)(q % w);
  T v = in[(size_t)old_of_new[n] * w + k];
  if constexpr (std::is_signed<T>::value) {   // node indices (signed, -1: none) are renumbered; flags are copied
    if (remap && v >= 0) v = (T)new_of_old[(int)v];
  }
  out[q] = v;
}

template <typename T>
int permute_rows(cudaStream_t s, int nn, int w, const int* d_oon, const int* d_noo, T*& p, bool remap) {
  if (!p || w == 0) return ASR_OK;
  T* q = nullptr;
  ASR_CUDA(cudaMalloc(&q, std::max<size_t>((size_t)nn * w, 1) * sizeof(T)));
  long n = (long)nn * w;
  k_perm_rows<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(nn, w, d_oon, d_noo, p, q, remap);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaFree(q);
    set_error("permute_rows: %s", cudaGetErrorString(e));
    return ASR_ECUDA;
  }
  cudaFree(p);
  p = q;
  return ASR_OK;
}

// reverse Cuthill-McKee order of the symmetrised hop graph (host; components in order of their lowest node, each from a
// pseudo-peripheral node of minimum degree), with node 0 moved to the front
static std::vector<int> rcm_order(int nn, int ns, const std::vector<int>& hopr) {
  std::vector<std::vector<int>> adj(nn);
  for (int i = 0; i < nn; ++i)
    for (int k = 0; k < ns; ++k) {
      int j = hopr[(size_t)i * ns + k];
      if (j >= 0 && j != i) { adj[i].push_back(j); adj[j].push_back(i); }
    }
  for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
  std::vector<int> deg(nn), order, level(nn, -1);
  for (int i = 0; i < nn; ++i) deg[i] = (int)adj[i].size();
  order.reserve(nn);
  std::vector<char> seen(nn, 0);
  auto bfs_far = [&](int s0, std::vector<int>& comp) {   // breadth-first levels; returns a last-level node of min degree
    comp.clear();
    comp.push_back(s0);
    level[s0] = 0;
    for (size_t h = 0; h < comp.size(); ++h)
      for (int j : adj[comp[h]]) if (level[j] < 0) { level[j] = level[comp[h]] + 1; comp.push_back(j); }
    int far = comp.back(), lmax = level[far];
    for (int v : comp) if (level[v] == lmax && deg[v] < deg[far]) far = v;
    for (int v : comp) level[v] = -1;
    return std::make_pair(far, lmax);
  };
  std::vector<int> comp;
  for (int r = 0; r < nn; ++r) {
    if (seen[r]) continue;
    int s0 = r, ecc = -1;
    for (int it = 0; it < 8; ++it) {   // pseudo-peripheral node: move to the far end while the eccentricity grows
      auto fe = bfs_far(s0, comp);
      if (fe.second <= ecc) break;
      ecc = fe.second;
      s0 = fe.first;
    }
    size_t base = order.size();
    order.push_back(s0);
    seen[s0] = 1;
    for (size_t h = base; h < order.size(); ++h) {
      int v = order[h];
      std::vector<int> nb;
      for (int j : adj[v]) if (!seen[j]) { seen[j] = 1; nb.push_back(j); }
      std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
      order.insert(order.end(), nb.begin(), nb.end());
    }
  }
  std::reverse(order.begin(), order.end());
  std::vector<int> out;
  out.reserve(nn);
  out.push_back(0);
  for (int v : order) if (v != 0) out.push_back(v);
  return out;
}

int reorder_nodes(asr_ctx* ctx, asr_op* op) {
  cudaStream_t s = ctx->stream;
  const int nn = op->nn, ns = op->nslot, nsm = op->nsmax;
  std::vector<int> hr((size_t)nn * std::max(ns, 1), -1);
  if (ns) ASR_CUDA(cudaMemcpyAsync(hr.data(), op->d_hopr, (size_t)nn * ns * sizeof(int), cudaMemcpyDeviceToHost, s));
  std::vector<int> sp(nn + 1);
  std::vector<uint8_t> sb(std::max(op->nstab, 1));
  ASR_CUDA(cudaMemcpyAsync(sp.data(), op->d_stab_ptr, (nn + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (op->nstab) ASR_CUDA(cudaMemcpyAsync(sb.data(), op->d_stab, op->nstab, cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  std::vector<int> oon = rcm_order(nn, ns, hr), noo(nn);
  for (int n = 0; n < nn; ++n) noo[oon[n]] = n;
  int *d_oon = nullptr, *d_noo = nullptr;
  if (cudaMalloc(&d_oon, nn * sizeof(int)) != cudaSuccess || cudaMalloc(&d_noo, nn * sizeof(int)) != cudaSuccess ||
      cudaMemcpyAsync(d_oon, oon.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(d_noo, noo.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess) {
    cudaFree(d_oon);
    cudaFree(d_noo);
    set_error("reorder_nodes: device allocation or copy of the node order failed");
    return ASR_ENOMEM;
  }
  int rc = ASR_OK;
  auto run = [&](int r) { if (rc == ASR_OK) rc = r; };
  run(permute_rows<int>(s, nn, 1, d_oon, d_noo, op->d_site, false));
  run(permute_rows<int>(s, nn, 1, d_oon, d_noo, op->d_level, false));
  run(permute_rows<int>(s, nn, 1, d_oon, d_noo, op->d_orb, false));
  run(permute_rows<int8_t>(s, nn, 1, d_oon, d_noo, op->d_lst, false));
  run(permute_rows<int8_t>(s, nn, 1, d_oon, d_noo, op->d_ncl, false));
  run(permute_rows<int8_t>(s, nn, 1, d_oon, d_noo, op->d_typ, false));
  run(permute_rows<int8_t>(s, nn, 1, d_oon, d_noo, op->d_start, false));
  run(permute_rows<int8_t>(s, nn, 1, d_oon, d_noo, op->d_frozen, false));
  run(permute_rows<double>(s, nn, 1, d_oon, d_noo, op->d_sq, false));
  run(permute_rows<double>(s, nn, 1, d_oon, d_noo, op->d_isq, false));
  run(permute_rows<int>(s, nn, nsm, d_oon, d_noo, op->d_flipr, true));
  run(permute_rows<uint8_t>(s, nn, nsm, d_oon, d_noo, op->d_flipg, false));
  run(permute_rows<int>(s, nn, ns, d_oon, d_noo, op->d_hopr, true));
  run(permute_rows<uint8_t>(s, nn, ns, d_oon, d_noo, op->d_hopg, false));
  cudaFree(d_oon);
  cudaFree(d_noo);
  if (rc != ASR_OK) return rc;
  // stabiliser lists (ragged): rebuilt on the host in the new order
  std::vector<int> sp2(nn + 1, 0);
  std::vector<uint8_t> sb2(std::max(op->nstab, 1));
  for (int n = 0; n < nn; ++n) {
    int o = oon[n], len = sp[o + 1] - sp[o];
    sp2[n + 1] = sp2[n] + len;
    std::copy(sb.begin() + sp[o], sb.begin() + sp[o] + len, sb2.begin() + sp2[n]);
  }
  ASR_CUDA(cudaMemcpyAsync(op->d_stab_ptr, sp2.data(), (nn + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
  if (op->nstab) ASR_CUDA(cudaMemcpyAsync(op->d_stab, sb2.data(), op->nstab, cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  op->old_of_new = std::move(oon);
  op->new_of_old = std::move(noo);
  return ASR_OK;
}

int build_operator(asr_ctx* ctx, int nsite, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* cls,
                   const int* perm, int nop, int start, int maxlevel, int maxrank, const int* flippable, const int* stype,
                   asr_op* op, const int* tsite, int ntarget, int* tnode, int* tgop) {
  cudaStream_t s = ctx->stream;
  // ---- checks of the reference (src/asr_augcls.f90:620-637)
  for (int i = 0; i < nsite; ++i)
    if (perm[i] != i + 1) { set_error("build_augcls_operator: operation 1 must be the identity"); return ASR_EINVAL; }
  if (start < 1 || start > nsite) { set_error("build_augcls_operator: start site out of range"); return ASR_EINVAL; }
  for (int g = 0; g < nop; ++g) {
    const int* p = perm + (size_t)g * nsite;
    if (p[start - 1] != start) { set_error("build_augcls_operator: the group does not fix the start site"); return ASR_EINVAL; }
    for (int i = 0; i < nsite; ++i) {
      if (p[i] < 1 || p[i] > nsite) { set_error("build_augcls_operator: perm out of range"); return ASR_EINVAL; }
      if (cls[p[i] - 1] != cls[i]) { set_error("build_augcls_operator: an operation does not preserve the site classes"); return ASR_EINVAL; }
    }
  }
  if (nop > 255) { set_error("build_augcls_operator: at most 255 operations"); return ASR_EINVAL; }
  int nsm = 0;
  for (int k = 0; k < ncls; ++k) nsm = std::max(nsm, nsc[k]);
  std::vector<int> nst(nsite);
  int nflip = 0;
  int maxdeg = 0;
  for (int r = 0; r < nsite; ++r) {
    bool cf = flippable ? flippable[r] != 0 : true;
    nst[r] = cf ? nsc[cls[r] - 1] : 1;
    if (nst[r] > 1) ++nflip;
    maxdeg = std::max(maxdeg, nbr_ptr[r + 1] - nbr_ptr[r]);
  }
  long rk = maxrank > 0 ? maxrank : LONG_MAX;
  rk = std::min<long>(rk, 3L * std::max(maxlevel, 0));
  rk = std::min<long>(rk, nflip);
  int R = (int)std::max<long>(rk, 1);
  if (R > RMAX) { set_error("build_augcls_operator: rank %d above the device key width %d (set maxrank)", R, RMAX); return ASR_EINVAL; }
  const int W = R + 1;
  const int rkmax = maxrank > 0 ? maxrank : INT_MAX;
  // ---- device inputs
  DBuf<int> d_nbr_ptr, d_nbr, d_perm, d_nst, d_cls, d_nsc, d_canflip, d_stype;
  ASR_TRY(d_nbr_ptr.alloc(nsite + 1));
  ASR_TRY(d_nbr.alloc(std::max(nbr_ptr[nsite] - 1, 1)));
  ASR_TRY(d_perm.alloc((size_t)nsite * nop));
  ASR_TRY(d_nst.alloc(nsite)); ASR_TRY(d_cls.alloc(nsite)); ASR_TRY(d_nsc.alloc(ncls));
  ASR_TRY(d_canflip.alloc(nsite)); ASR_TRY(d_stype.alloc(nsite));
  std::vector<int> cf(nsite), st(nsite);
  for (int r = 0; r < nsite; ++r) { cf[r] = flippable ? (flippable[r] != 0) : 1; st[r] = stype ? stype[r] : 1; }
  ASR_CUDA(cudaMemcpyAsync(d_nbr_ptr.p, nbr_ptr, (nsite + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_nbr.p, nbr, (nbr_ptr[nsite] - 1) * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_perm.p, perm, (size_t)nsite * nop * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_nst.p, nst.data(), nsite * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_cls.p, cls, nsite * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_nsc.p, nsc, ncls * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_canflip.p, cf.data(), nsite * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_stype.p, st.data(), nsite * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
  BuildView B{nsite, nop, nsm, W, R, rkmax, maxdeg, d_nbr_ptr.p, d_nbr.p, d_perm.p, d_nst.p};

  // ---- start node: the start site with the reference configuration (its orbit must be 1)
  for (int g = 0; g < nop; ++g) if (perm[(size_t)g * nsite + start - 1] != start) { set_error("build_augcls_operator: start site is not invariant under the group"); return ASR_EINVAL; }
  size_t cap = 1 << 16;
  DBuf<int> nkey, nlevel, norb;
  ASR_TRY(nkey.alloc(cap * W)); ASR_TRY(nlevel.alloc(cap)); ASR_TRY(norb.alloc(cap));
  {
    std::vector<int> k0(W, INT_MAX);
    k0[0] = start;
    int z = 0, one = 1;
    ASR_CUDA(cudaMemcpyAsync(nkey.p, k0.data(), W * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(nlevel.p, &z, sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(norb.p, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaStreamSynchronize(s));
  }
  uint32_t tcap = 1u << 16;
  DBuf<int> table;
  ASR_TRY(table.alloc(tcap));
  ASR_CUDA(cudaMemsetAsync(table.p, 0xff, tcap * sizeof(int), s));
  k_rehash<<<1, 32, 0, s>>>(1, W, nkey.p, table.p, tcap - 1, ctx->d_err);
  int nn = 1;
  DBuf<int> cnt, off, ckey, cosz, first, pos, slot;
  DBuf<signed char> cstat;
  DBuf<unsigned char> tmp;
  const int T1 = maxdeg + 1, T2 = T1 * T1;
  const long CH = std::min<long>(1L << 25, (long)(INT_MAX / 2) / W);   // candidates per chunk
  int lo = 0, hi = 1;
  for (int lev = 0; lev < maxlevel && lo < hi; ++lev) {
    int a = lo;
    int nb_nodes = std::max(1, (int)std::min<long>(hi - lo, CH / std::max(T2, 1)));
    while (a < hi) {
      int b = std::min(hi, a + nb_nodes);
      long ntrip;
      int C;
      for (;;) {
        ntrip = (long)(b - a) * T2;
        ASR_TRY(cnt.alloc(ntrip + 1)); ASR_TRY(off.alloc(ntrip + 1));
        k_count<<<blocks(ntrip, 256), 256, 0, s>>>(B, nkey.p, a, (int)ntrip, cnt.p, ctx->d_err);
        ASR_CUDA(cudaMemsetAsync(cnt.p + ntrip, 0, sizeof(int), s));
        ASR_TRY(exclusive_scan(cnt.p, off.p, (int)ntrip + 1, tmp, s));
        ASR_CUDA(cudaMemcpyAsync(&C, off.p + ntrip, sizeof(int), cudaMemcpyDeviceToHost, s));
        ASR_TRY(check_err(ctx, "count"));
        if (C <= CH || b - a == 1) break;
        b = a + (b - a) / 2;
      }
      if (C > 0) {
        ASR_TRY(ckey.alloc((size_t)C * W)); ASR_TRY(cosz.alloc(C)); ASR_TRY(cstat.alloc(C));
        ASR_TRY(first.alloc(C + 1)); ASR_TRY(pos.alloc(C + 1)); ASR_TRY(slot.alloc(C));
        k_generate<<<blocks(ntrip, 128), 128, 0, s>>>(B, nkey.p, a, (int)ntrip, off.p, ckey.p, cosz.p, cstat.p, ctx->d_err);
        // table capacity: every node plus every pending candidate, load factor <= 1/2
        size_t need = (size_t)nn + (size_t)C;
        if ((size_t)tcap < 2 * need) {
          uint32_t nt = tcap;
          while ((size_t)nt < 2 * need) nt <<= 1;
          if (nt > (1u << 31)) { set_error("build_augcls_operator: node table above 2^31 entries"); return ASR_ENOMEM; }
          tcap = nt;
          ASR_TRY(table.alloc(tcap));
          ASR_CUDA(cudaMemsetAsync(table.p, 0xff, (size_t)tcap * sizeof(int), s));
          k_rehash<<<blocks(nn, 256), 256, 0, s>>>(nn, W, nkey.p, table.p, tcap - 1, ctx->d_err);
        }
        k_insert<<<blocks(C, 256), 256, 0, s>>>(C, W, ckey.p, cstat.p, nkey.p, table.p, tcap - 1, ctx->d_err);
        k_first<<<blocks(C, 256), 256, 0, s>>>(C, W, ckey.p, cstat.p, table.p, tcap - 1, first.p, slot.p, ctx->d_err);
        ASR_CUDA(cudaMemsetAsync(first.p + C, 0, sizeof(int), s));
        ASR_TRY(exclusive_scan(first.p, pos.p, C + 1, tmp, s));
        int nnew = 0;
        ASR_CUDA(cudaMemcpyAsync(&nnew, pos.p + C, sizeof(int), cudaMemcpyDeviceToHost, s));
        ASR_TRY(check_err(ctx, "insert"));
        if ((size_t)(nn + nnew) > cap) {
          size_t nc = cap;
          while (nc < (size_t)(nn + nnew)) nc *= 2;
          ASR_TRY(nkey.grow_keep(nc * W, s)); ASR_TRY(nlevel.grow_keep(nc, s)); ASR_TRY(norb.grow_keep(nc, s));
          cap = nc;
        }
        k_commit<<<blocks(C, 256), 256, 0, s>>>(C, W, ckey.p, cosz.p, first.p, pos.p, slot.p, nn, lev + 1, nkey.p, nlevel.p,
                                                norb.p, table.p);
        nn += nnew;
      }
      a = b;
    }
    lo = hi;
    hi = nn;
  }
  ASR_TRY(check_err(ctx, "closure"));
  // ---- node tables
  int nslot = maxdeg;
  DBuf<int> scnt, sptr;
  ASR_TRY(scnt.alloc(nn + 1)); ASR_TRY(sptr.alloc(nn + 1));
  k_stab_count<<<blocks(nn, 128), 128, 0, s>>>(B, nn, nkey.p, norb.p, scnt.p, ctx->d_err);
  ASR_CUDA(cudaMemsetAsync(scnt.p + nn, 0, sizeof(int), s));
  ASR_TRY(exclusive_scan(scnt.p, sptr.p, nn + 1, tmp, s));
  int nstab = 0;
  ASR_CUDA(cudaMemcpyAsync(&nstab, sptr.p + nn, sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_TRY(check_err(ctx, "stabilisers"));
  DBuf<int> site, flipr, hopr;
  DBuf<int8_t> lst, ncl, typ, stt, frz;
  DBuf<double> sq, isq;
  DBuf<uint8_t> flipg, hopg, stab;
  ASR_TRY(site.alloc(nn)); ASR_TRY(lst.alloc(nn)); ASR_TRY(ncl.alloc(nn)); ASR_TRY(typ.alloc(nn)); ASR_TRY(stt.alloc(nn));
  ASR_TRY(frz.alloc(nn)); ASR_TRY(sq.alloc(nn)); ASR_TRY(isq.alloc(nn));
  ASR_TRY(flipr.alloc((size_t)nsm * nn)); ASR_TRY(flipg.alloc((size_t)nsm * nn));
  ASR_TRY(hopr.alloc((size_t)std::max(nslot, 1) * nn)); ASR_TRY(hopg.alloc((size_t)std::max(nslot, 1) * nn));
  ASR_TRY(stab.alloc(std::max(nstab, 1)));
  ASR_CUDA(cudaMemsetAsync(frz.p, 0, nn, s));
  TableOut T{site.p, lst.p, ncl.p, typ.p, stt.p, sq.p, isq.p, flipr.p, flipg.p, hopr.p, hopg.p, sptr.p, stab.p};
  k_tables<<<blocks(nn, 128), 128, 0, s>>>(B, nn, nslot, nkey.p, norb.p, table.p, tcap - 1, d_cls.p, d_nsc.p, d_canflip.p,
                                           d_stype.p, start, T);
  ASR_TRY(check_err(ctx, "tables"));
  if (tsite && ntarget > 0) {
    for (int t = 0; t < ntarget; ++t)
      if (tsite[t] < 1 || tsite[t] > nsite) { set_error("build_augcls_operator: target site out of range"); return ASR_EINVAL; }
    const int nq = ntarget * nsm;
    DBuf<int> d_ts, d_tn, d_tg;
    ASR_TRY(d_ts.alloc(ntarget)); ASR_TRY(d_tn.alloc(nq)); ASR_TRY(d_tg.alloc(nq));
    ASR_CUDA(cudaMemcpyAsync(d_ts.p, tsite, ntarget * sizeof(int), cudaMemcpyHostToDevice, s));
    k_targets<<<blocks(nq, 128), 128, 0, s>>>(B, ntarget, d_ts.p, nkey.p, table.p, tcap - 1, d_cls.p, d_nsc.p, d_canflip.p,
                                             start, d_tn.p, d_tg.p);
    ASR_CUDA(cudaMemcpyAsync(tnode, d_tn.p, nq * sizeof(int), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaMemcpyAsync(tgop, d_tg.p, nq * sizeof(int), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    ASR_TRY(check_err(ctx, "targets"));
  }
  ASR_CUDA(cudaGetLastError());
  op->nn = nn; op->nslot = nslot; op->nsmax = nsm; op->nop = nop; op->ncls = ncls; op->nsite = nsite; op->nstab = nstab;
  op->start_site = start;
  op->d_site = site.release(); op->d_level = nlevel.release(); op->d_orb = norb.release();
  op->d_lst = lst.release(); op->d_ncl = ncl.release(); op->d_typ = typ.release(); op->d_start = stt.release();
  op->d_frozen = frz.release(); op->d_sq = sq.release(); op->d_isq = isq.release();
  op->d_flipr = flipr.release(); op->d_flipg = flipg.release(); op->d_hopr = hopr.release(); op->d_hopg = hopg.release();
  op->d_stab_ptr = sptr.release(); op->d_stab = stab.release();
  const char* order_env = getenv("ASR_NODE_ORDER");   // "build": keep the reference numbering on the device
  if (!(order_env && std::string(order_env) == "build")) ASR_TRY(reorder_nodes(ctx, op));
  return ASR_OK;
}

}  // namespace asrb
