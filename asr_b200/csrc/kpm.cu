// Kernel polynomial method on an explicit supercell: kpm_moments / kpm_dos (src/reference/asr_kpm.f90:39-87) on the
// realisation operator lmto_real_op (src/reference/asr_lmto_realization.f90:120-191), generalised to n species.
//
// Layout: the nvec random vectors are the innermost index, x[(site * 9 + l) * V + v] with V = 64, so one block row of
// 64 threads covers one site of every vector and each orbital load is coalesced.  The bond blocks sit in shared
// memory; d and c per species are tiny tables there too.  One Chebyshev step is one kernel:
//     t_{n+1} = 2 (H t_n - cen t_n) / sc - t_{n-1}   (n = 0: t_1 = (H t_0 - cen t_0) / sc),  H = e + c + d S d  (o = 0)
// with the FP64 partial dots r . t_{n+1}, t_{n+1} . t_{n+1} and t_{n+1} . t_n per vector.  The Rademacher vectors r are
// regenerated from a counter-based hash (splitmix64) instead of being read.  Two moment sets come out of one matvec
// with the Chebyshev doubling identities mu_2n = 2 <t_n|t_n> - mu_0, mu_2n+1 = 2 <t_n+1|t_n> - mu_1 (H symmetric), or
// one moment per matvec as the reference does (mu_n = <r|t_n>).
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "op.h"

struct asr_supercell {
  asr_ctx* ctx = nullptr;
  int n = 0, ns = 0, nsp = 0;
  bool o_zero = true, e_zero = true;
  int* d_nbr = nullptr;          // (ns, n) 0-based
  uint8_t* d_spc = nullptr;      // (n) 0-based species
  double* d_par = nullptr;       // c, d, o, e: 4 x (9, nsp)
  std::vector<double> par_h;     // host copy of the same
  double* d_blocks = nullptr;    // [1 + ns][l][l']
  float* d_blocks_f = nullptr;
};

namespace asrb {
namespace {

constexpr int KV = 64;           // vectors per site row
constexpr int KSITES = 4;        // sites per 256-thread block row

__host__ __device__ inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
// Rademacher entry q of vector v: +1 if bit 63 of splitmix64(seed * phi + (v << 40) + q) is clear
__device__ __forceinline__ double rademacher(uint64_t seed, uint64_t v, uint64_t q) {
  return (splitmix64(seed * 0x9E3779B97F4A7C15ULL + (v << 40) + q) >> 63) ? -1.0 : 1.0;
}

template <typename ST> __device__ __forceinline__ ST fma_t(ST a, ST b, ST c);
template <> __device__ __forceinline__ double fma_t<double>(double a, double b, double c) { return fma(a, b, c); }
template <> __device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return fmaf(a, b, c); }

struct ScView {
  int n, ns, nsp;
  const int* nbr;
  const uint8_t* spc;
  const double* par;   // c | d | o | e, each (9, nsp)
};

// y = h x = c x + d S (d x) for one (site, vector): acc over the on-site and ns bond blocks
template <typename ST>
__device__ __forceinline__ void h_site(const ScView& S, const ST* Bs, const double* ps, const ST* x, int i, int v, double* y) {
  ST acc[9];
  for (int l = 0; l < 9; ++l) acc[l] = (ST)0;
  int si = S.spc[i];
  {
    ST u[9];
    for (int l = 0; l < 9; ++l) u[l] = (ST)ps[9 * S.nsp + l + 9 * si] * x[((size_t)i * 9 + l) * KV + v];
    for (int l = 0; l < 9; ++l)
      for (int lp = 0; lp < 9; ++lp) acc[l] = fma_t<ST>(Bs[l * 9 + lp], u[lp], acc[l]);
  }
  for (int k = 0; k < S.ns; ++k) {
    int j = S.nbr[k + (size_t)S.ns * i];
    int sj = S.spc[j];
    const ST* Bk = Bs + (size_t)(k + 1) * 81;
    ST u[9];
    for (int l = 0; l < 9; ++l) u[l] = (ST)ps[9 * S.nsp + l + 9 * sj] * x[((size_t)j * 9 + l) * KV + v];
    for (int l = 0; l < 9; ++l)
      for (int lp = 0; lp < 9; ++lp) acc[l] = fma_t<ST>(Bk[l * 9 + lp], u[lp], acc[l]);
  }
  for (int l = 0; l < 9; ++l)
    y[l] = ps[l + 9 * si] * (double)x[((size_t)i * 9 + l) * KV + v] + ps[9 * S.nsp + l + 9 * si] * (double)acc[l];
}

// smem: blocks [(1 + ns) * 81] (ST), then parameters 4 * 9 * nsp (double)
template <typename ST>
__device__ __forceinline__ void load_smem(const ScView& S, const ST* blocks, ST*& Bs, double*& ps) {
  extern __shared__ unsigned char sm_raw[];
  ps = (double*)sm_raw;
  Bs = (ST*)(ps + 4 * 9 * S.nsp);
  for (int q = threadIdx.x; q < 4 * 9 * S.nsp; q += blockDim.x) ps[q] = S.par[q];
  for (int q = threadIdx.x; q < (S.ns + 1) * 81; q += blockDim.x) Bs[q] = blocks[q];
  __syncthreads();
}

// one Chebyshev step, o = 0: t_new = 2 (H t - cen t)/sc - t_old (first: (H t - cen t)/sc); partial dots per vector:
// part[blk][v] = (r . t_new, t_new . t_new, t_new . t)
template <typename ST>
__global__ void __launch_bounds__(KSITES * KV) k_cheb(ScView S, const ST* __restrict__ blocks, const ST* __restrict__ t,
                                                      const ST* __restrict__ told, ST* __restrict__ tnew, double cen, double isc,
                                                      bool first, bool has_e, uint64_t seed, int v0, double* part) {
  ST* Bs;
  double* ps;
  load_smem<ST>(S, blocks, Bs, ps);
  const int v = threadIdx.x % KV, row = threadIdx.x / KV;
  double rt = 0.0, tt = 0.0, tp = 0.0;
  for (int i = blockIdx.x * KSITES + row; i < S.n; i += gridDim.x * KSITES) {
    double y[9];
    h_site<ST>(S, Bs, ps, t, i, v, y);
    int si = S.spc[i];
    for (int l = 0; l < 9; ++l) {
      size_t q = ((size_t)i * 9 + l) * KV + v;
      double tl = (double)t[q];
      double hy = y[l] + (has_e ? ps[27 * S.nsp + l + 9 * si] * tl : 0.0);
      double tn = first ? (hy - cen * tl) * isc : 2.0 * (hy - cen * tl) * isc - (double)told[q];
      ST ts = (ST)tn;
      tnew[q] = ts;
      double tr = (double)ts;
      rt += rademacher(seed, (uint64_t)(v0 + v), (uint64_t)i * 9 + l) * tr;
      tt += tr * tr;
      tp += tr * tl;
    }
  }
  __shared__ double red[KSITES][KV][3];
  red[row][v][0] = rt; red[row][v][1] = tt; red[row][v][2] = tp;
  __syncthreads();
  if (row == 0) {
    for (int r = 1; r < KSITES; ++r) { rt += red[r][v][0]; tt += red[r][v][1]; tp += red[r][v][2]; }
    double* out = part + ((size_t)blockIdx.x * KV + v) * 3;
    out[0] = rt; out[1] = tt; out[2] = tp;
  }
}

// acc += B[l][.] . x for one padded block row (12 entries, the last 3 zero): vector loads from shared memory.  The
// loads are volatile so that they stay next to their use: hoisting all 27 rows of a block ahead of the multiplies
// (what the compiler does otherwise) costs 80 registers a thread and halves the occupancy.
__device__ __forceinline__ float4 lds_f4(const float* p) {
  float4 r;
  unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.volatile.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w) : "r"(a));
  return r;
}
__device__ __forceinline__ double2 lds_d2(const double* p) {
  double2 r;
  unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.volatile.shared.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "r"(a));
  return r;
}
__device__ __forceinline__ float row9(const float* __restrict__ row, const float* x, float acc) {
  float4 a = lds_f4(row), b = lds_f4(row + 4), c = lds_f4(row + 8);
  acc = fmaf(a.x, x[0], acc); acc = fmaf(a.y, x[1], acc); acc = fmaf(a.z, x[2], acc); acc = fmaf(a.w, x[3], acc);
  acc = fmaf(b.x, x[4], acc); acc = fmaf(b.y, x[5], acc); acc = fmaf(b.z, x[6], acc); acc = fmaf(b.w, x[7], acc);
  return fmaf(c.x, x[8], acc);
}
__device__ __forceinline__ double row9(const double* __restrict__ row, const double* x, double acc) {
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    double2 a = lds_d2(row + 2 * q);
    acc = fma(a.x, x[2 * q], acc);
    if (q < 4) acc = fma(a.y, x[2 * q + 1], acc);
  }
  return acc;
}
constexpr int KRW = 12;   // padded block row (16-byte aligned)

// Chebyshev step for o = 0 on d-scaled vectors u = d o t (per site and orbital, d of the site's species): with
// h t = c t + d S (d t), the recurrence t' = 2 (H t - cen t) / sc - t_old becomes
//   u' = 2 ((c + e - cen) o u + d^2 o S u) / sc - u_old,
// so the gathered neighbour rows need neither their species nor a scaling.  Partial dots of t (weights 1/d^2, 1/d):
// part[blk][v] = (r . t', t' . t', t' . t).  The next slot's neighbour index and row are loaded while the current slot
// is multiplied.
struct UCoef {
  const double* cc;   // (c + e - cen) per (orbital, species)
  const double* d2;   // d^2
  const double* w2;   // 1 / d^2
  const double* w1;   // 1 / d
};

template <typename ST, bool WANT_R>
__global__ void __launch_bounds__(KSITES * KV, sizeof(ST) == 8 ? 3 : 0) k_cheb_u(ScView S, const ST* __restrict__ blocks, const double* __restrict__ coef,
                                                        const ST* __restrict__ u, const ST* __restrict__ uold,
                                                        ST* __restrict__ unew, double isc, bool first, uint64_t seed, int v0,
                                                        double* part) {
  extern __shared__ unsigned char sm_raw[];
  const int np = 9 * S.nsp;
  double* cs = (double*)sm_raw;                 // cc | d2 | w2 | w1
  ST* Bs = (ST*)(cs + 4 * np);                  // [1 + ns][9][KRW]
  for (int q = threadIdx.x; q < 4 * np; q += blockDim.x) cs[q] = coef[q];
  for (int q = threadIdx.x; q < (S.ns + 1) * 9 * KRW; q += blockDim.x) {
    int c = q % KRW, r = q / KRW;
    Bs[q] = c < 9 ? blocks[r * 9 + c] : (ST)0;
  }
  __syncthreads();
  const int v = threadIdx.x % KV, row = threadIdx.x / KV;
  double rt = 0.0, tt = 0.0, tp = 0.0;
  for (int i = blockIdx.x * KSITES + row; i < S.n; i += gridDim.x * KSITES) {
    ST acc[9], xa[9], xb[9], uo[9];
    for (int l = 0; l < 9; ++l) acc[l] = (ST)0;
    const ST* ui = u + (size_t)i * 9 * KV + v;
    for (int l = 0; l < 9; ++l) uo[l] = ui[l * KV];
    const int* nb = S.nbr + (size_t)S.ns * i;
    int jn = S.ns > 0 ? nb[0] : 0;
    if (S.ns > 0) { const ST* src = u + (size_t)jn * 9 * KV + v; for (int l = 0; l < 9; ++l) xa[l] = src[l * KV]; }
    // on-site block
    for (int l = 0; l < 9; ++l) acc[l] = row9(Bs + l * KRW, uo, acc[l]);
#pragma unroll 1
    for (int k = 0; k < S.ns; ++k) {
      if (k + 1 < S.ns) {
        jn = nb[k + 1];
        const ST* src = u + (size_t)jn * 9 * KV + v;
        for (int l = 0; l < 9; ++l) xb[l] = src[l * KV];
      }
      const ST* Bk = Bs + (size_t)(k + 1) * 9 * KRW;
      for (int l = 0; l < 9; ++l) acc[l] = row9(Bk + l * KRW, xa, acc[l]);
      for (int l = 0; l < 9; ++l) xa[l] = xb[l];
    }
    const int si = S.spc[i];
    ST* uni = unew + (size_t)i * 9 * KV + v;
    const ST* uoi = first ? nullptr : uold + (size_t)i * 9 * KV + v;
    for (int l = 0; l < 9; ++l) {
      const int q = l + 9 * si;
      double y = cs[q] * (double)uo[l] + cs[np + q] * (double)acc[l];
      double un = first ? y * isc : 2.0 * y * isc - (double)uoi[l * KV];
      ST us = (ST)un;
      uni[l * KV] = us;
      double ur = (double)us;
      tt += cs[2 * np + q] * ur * ur;
      tp += cs[2 * np + q] * ur * (double)uo[l];
      if (WANT_R) rt += rademacher(seed, (uint64_t)(v0 + v), (uint64_t)i * 9 + l) * ur * cs[3 * np + q];
    }
  }
  __shared__ double red[KSITES][KV][3];
  red[row][v][0] = rt; red[row][v][1] = tt; red[row][v][2] = tp;
  __syncthreads();
  if (row == 0) {
    for (int r = 1; r < KSITES; ++r) { rt += red[r][v][0]; tt += red[r][v][1]; tp += red[r][v][2]; }
    double* out = part + ((size_t)blockIdx.x * KV + v) * 3;
    out[0] = rt; out[1] = tt; out[2] = tp;
  }
}

// u_0 = d o r (d of each site's species)
template <typename ST>
__global__ void k_rademacher_init_scaled(ScView S, uint64_t seed, int v0, ST* t) {
  size_t tot = (size_t)S.n * 9 * KV;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x) {
    int v = (int)(q % KV);
    size_t e = q / KV;   // site * 9 + l
    int site = (int)(e / 9), l = (int)(e % 9);
    double d = S.par[9 * S.nsp + l + 9 * S.spc[site]];
    t[q] = (ST)(d * rademacher(seed, (uint64_t)(v0 + v), (uint64_t)e));
  }
}

// general operator (o != 0): w = h x (stored, FP64 math, ST storage)
template <typename ST>
__global__ void __launch_bounds__(KSITES * KV) k_h(ScView S, const ST* __restrict__ blocks, const ST* __restrict__ x,
                                                   bool oscale, ST* __restrict__ w) {
  ST* Bs;
  double* ps;
  load_smem<ST>(S, blocks, Bs, ps);
  const int v = threadIdx.x % KV, row = threadIdx.x / KV;
  for (int i = blockIdx.x * KSITES + row; i < S.n; i += gridDim.x * KSITES) {
    double y[9];
    h_site<ST>(S, Bs, ps, x, i, v, y);
    int si = S.spc[i];
    for (int l = 0; l < 9; ++l) {
      double f = oscale ? ps[18 * S.nsp + l + 9 * si] : 1.0;   // o h x when requested
      w[((size_t)i * 9 + l) * KV + v] = (ST)(f * y[l]);
    }
  }
}

// general Chebyshev combination: y = e t + w1 - w3 (w1 = h t, w3 = h o h t)
template <typename ST>
__global__ void __launch_bounds__(KSITES * KV) k_cheb_comb(ScView S, const ST* __restrict__ t, const ST* __restrict__ w1,
                                                           const ST* __restrict__ w3, const ST* __restrict__ told,
                                                           ST* __restrict__ tnew, double cen, double isc, bool first,
                                                           uint64_t seed, int v0, double* part) {
  const int v = threadIdx.x % KV, row = threadIdx.x / KV;
  double rt = 0.0, tt = 0.0, tp = 0.0;
  for (int i = blockIdx.x * KSITES + row; i < S.n; i += gridDim.x * KSITES) {
    int si = S.spc[i];
    for (int l = 0; l < 9; ++l) {
      size_t q = ((size_t)i * 9 + l) * KV + v;
      double tl = (double)t[q];
      double hy = S.par[27 * S.nsp + l + 9 * si] * tl + (double)w1[q] - (double)w3[q];
      double tn = first ? (hy - cen * tl) * isc : 2.0 * (hy - cen * tl) * isc - (double)told[q];
      ST ts = (ST)tn;
      tnew[q] = ts;
      double tr = (double)ts;
      rt += rademacher(seed, (uint64_t)(v0 + v), (uint64_t)i * 9 + l) * tr;
      tt += tr * tr;
      tp += tr * tl;
    }
  }
  __shared__ double red[KSITES][KV][3];
  red[row][v][0] = rt; red[row][v][1] = tt; red[row][v][2] = tp;
  __syncthreads();
  if (row == 0) {
    for (int r = 1; r < KSITES; ++r) { rt += red[r][v][0]; tt += red[r][v][1]; tp += red[r][v][2]; }
    double* out = part + ((size_t)blockIdx.x * KV + v) * 3;
    out[0] = rt; out[1] = tt; out[2] = tp;
  }
}

template <typename ST>
__global__ void k_rademacher_init(int n, uint64_t seed, int v0, ST* t) {
  size_t tot = (size_t)n * 9 * KV;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x) {
    int v = (int)(q % KV);
    size_t e = q / KV;   // site * 9 + l
    t[q] = (ST)rademacher(seed, (uint64_t)(v0 + v), (uint64_t)e);
  }
}

// sum of the block partials per vector in a fixed order: out[v][3]
__global__ void k_kpm_reduce(const double* part, int nblk, double* out) {
  int v = threadIdx.x;
  if (v >= KV) return;
  double a = 0, b = 0, c = 0;
  for (int q = 0; q < nblk; ++q) {
    const double* p = part + ((size_t)q * KV + v) * 3;
    a += p[0]; b += p[1]; c += p[2];
  }
  out[v * 3 + 0] = a; out[v * 3 + 1] = b; out[v * 3 + 2] = c;
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  int alloc(size_t n) {
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      set_error("kpm: device allocation of %zu bytes failed", n * sizeof(T));
      return ASR_ENOMEM;
    }
    return ASR_OK;
  }
};

template <typename ST>
int kpm_run(asr_ctx* ctx, asr_supercell* sc, double cen, double scl, int nmom, int v0, int nvec, uint64_t seed, bool doubling,
            double* mu) {
  cudaStream_t s = ctx->stream;
  const int n = sc->n;
  ScView S{n, sc->ns, sc->nsp, sc->d_nbr, sc->d_spc, sc->d_par};
  const ST* blocks = std::is_same<ST, double>::value ? (const ST*)sc->d_blocks : (const ST*)sc->d_blocks_f;
  const size_t nel = (size_t)n * 9 * KV;
  const size_t smem = 4 * 9 * sc->nsp * sizeof(double) + (size_t)(sc->ns + 1) * 81 * sizeof(ST);
  const int grid = ctx->num_sms * 4;
  const bool general = !sc->o_zero;
  DevBuf<ST> T0, T1, T2, W1, W2, W3;
  ASR_TRY(T0.alloc(nel)); ASR_TRY(T1.alloc(nel)); ASR_TRY(T2.alloc(nel));
  if (general) { ASR_TRY(W1.alloc(nel)); ASR_TRY(W2.alloc(nel)); ASR_TRY(W3.alloc(nel)); }
  DevBuf<double> part, red;
  ASR_TRY(part.alloc((size_t)grid * KV * 3));
  // all reduced dots of the run: (nsteps, KV, 3)
  const int nsteps = doubling ? std::max(1, (nmom + 1) / 2) : std::max(1, nmom - 1);
  ASR_TRY(red.alloc((size_t)nsteps * KV * 3));
  for (int m = 0; m < nmom; ++m) mu[m] = 0.0;
  const double isc = 1.0 / scl;
  const double dim = 9.0 * n;
  std::vector<double> hred((size_t)nsteps * KV * 3);
  // coefficients of the d-scaled recurrence (o = 0): c + e - cen, d^2, 1/d^2, 1/d per (orbital, species)
  DevBuf<double> ucoef;
  const size_t smem_u = 4 * 9 * sc->nsp * sizeof(double) + (size_t)(sc->ns + 1) * 9 * KRW * sizeof(ST);
  bool dpos = true;
  if (!general) {
    const int np = 9 * sc->nsp;
    std::vector<double> hc(4 * (size_t)np);
    for (int q = 0; q < np; ++q) {
      double c = sc->par_h[q], d = sc->par_h[np + q], e = sc->par_h[3 * np + q];
      if (d == 0.0) dpos = false;
      hc[q] = c + e - cen;
      hc[np + q] = d * d;
      hc[2 * np + q] = d != 0.0 ? 1.0 / (d * d) : 0.0;
      hc[3 * np + q] = d != 0.0 ? 1.0 / d : 0.0;
    }
    if (dpos) {
      ASR_TRY(ucoef.alloc(hc.size()));
      ASR_CUDA(cudaMemcpyAsync(ucoef.p, hc.data(), hc.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    }
  }
  const bool scaled = !general && dpos;
  for (int vb = 0; vb < nvec; vb += KV) {
    const int nv = std::min(KV, nvec - vb);
    if (scaled) k_rademacher_init_scaled<ST><<<ctx->num_sms * 8, 256, 0, s>>>(S, seed, v0 + vb, T0.p);
    else k_rademacher_init<ST><<<ctx->num_sms * 8, 256, 0, s>>>(n, seed, v0 + vb, T0.p);
    ST *ta = T0.p, *tb = T1.p, *tc = T2.p;   // t_{k-1}, t_k, t_{k+1}
    // step 0: t_1 = (H t_0 - cen t_0) / sc
    for (int k = 0; k < nsteps; ++k) {
      const ST* tin = (k == 0) ? ta : tb;
      const ST* told = (k == 0) ? nullptr : ta;
      ST* tout = (k == 0) ? tb : tc;
      const int ps = ctx->prof_start(s);
      if (scaled) {
        // <r|t> is needed for every step without doubling, and for mu_1 (step 0) with it
        if (!doubling || k == 0)
          k_cheb_u<ST, true><<<grid, KSITES * KV, smem_u, s>>>(S, blocks, ucoef.p, tin, told, tout, isc, k == 0, seed, v0 + vb, part.p);
        else
          k_cheb_u<ST, false><<<grid, KSITES * KV, smem_u, s>>>(S, blocks, ucoef.p, tin, told, tout, isc, k == 0, seed, v0 + vb, part.p);
      } else if (!general) {
        k_cheb<ST><<<grid, KSITES * KV, smem, s>>>(S, blocks, tin, told, tout, cen, isc, k == 0, !sc->e_zero, seed, v0 + vb, part.p);
      } else {
        k_h<ST><<<grid, KSITES * KV, smem, s>>>(S, blocks, tin, false, W1.p);
        k_h<ST><<<grid, KSITES * KV, smem, s>>>(S, blocks, tin, true, W2.p);    // o h t
        k_h<ST><<<grid, KSITES * KV, smem, s>>>(S, blocks, W2.p, false, W3.p);
        k_cheb_comb<ST><<<grid, KSITES * KV, 0, s>>>(S, tin, W1.p, W3.p, told, tout, cen, isc, k == 0, seed, v0 + vb, part.p);
      }
      {   // algorithmic work of one Chebyshev step: read t_k and t_{k-1}, write t_{k+1}, one species byte per site; flops
          // 2 x 81 x (1 + slots) per site and vector per S application (one for o = 0, three for the general operator)
        const double sapp = general ? 3.0 : 1.0;
        const double streams = general ? 9.0 : 3.0;
        ctx->prof_stop(s, ps, ASR_KERNEL_KPM, (double)n * (KV * streams * 9 * sizeof(ST) + 1.0),
                       sapp * (double)n * KV * 2.0 * 81.0 * (1 + sc->ns));
      }
      k_kpm_reduce<<<1, KV, 0, s>>>(part.p, grid, red.p + (size_t)k * KV * 3);
      if (k > 0) { ST* t_ = ta; ta = tb; tb = tc; tc = t_; }
    }
    ASR_CUDA(cudaGetLastError());
    ASR_CUDA(cudaMemcpyAsync(hred.data(), red.p, hred.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    // moments of the vectors of this block: step k produced t_{k+1}; dots (r.t_{k+1}, t_{k+1}.t_{k+1}, t_{k+1}.t_k)
    for (int v = 0; v < nv; ++v) {
      auto R = [&](int k, int c) { return hred[((size_t)k * KV + v) * 3 + c]; };
      double m0 = 1.0;   // <r|r> / dim for a Rademacher vector
      double m1 = R(0, 0) / dim;
      if (!doubling) {
        mu[0] += m0;
        if (nmom > 1) mu[1] += m1;
        for (int m = 2; m < nmom; ++m) mu[m] += R(m - 1, 0) / dim;
      } else {
        // t_0 . t_0 = dim, t_1 . t_0 = r . t_1
        mu[0] += m0;
        if (nmom > 1) mu[1] += m1;
        for (int m = 2; m < nmom; ++m) {
          int nh = m / 2;   // mu_2n = 2 t_n.t_n/dim - mu_0 ; mu_2n+1 = 2 t_n+1.t_n/dim - mu_1
          double val;
          if (m % 2 == 0) val = 2.0 * R(nh - 1, 1) / dim - m0;   // t_nh . t_nh is from step nh - 1
          else val = 2.0 * R(nh, 2) / dim - m1;                  // t_{nh+1} . t_nh from step nh
          mu[m] += val;
        }
      }
    }
  }
  for (int m = 0; m < nmom; ++m) mu[m] /= (double)nvec;
  return ASR_OK;
}

}  // namespace
}  // namespace asrb

using namespace asrb;

extern "C" {

int asr_supercell_build(asr_ctx* ctx, int nsite, int nslot, const int* nbr, const int* spc, int nsp, const double* c,
                        const double* d, const double* o, const double* e, const double* block, const double* block0,
                        asr_supercell** out) {
  if (!ctx || !out || !nbr || !spc || !c || !d || !block || nsite < 1 || nslot < 0 || nsp < 1 || nsp > 255) {
    set_error("asr_supercell_build: bad argument");
    return ASR_EINVAL;
  }
  *out = nullptr;
  for (size_t q = 0; q < (size_t)nslot * nsite; ++q)
    if (nbr[q] < 1 || nbr[q] > nsite) { set_error("asr_supercell_build: neighbour index out of range"); return ASR_EINVAL; }
  std::vector<uint8_t> sp(nsite);
  for (int i = 0; i < nsite; ++i) {
    if (spc[i] < 1 || spc[i] > nsp) { set_error("asr_supercell_build: species index out of range"); return ASR_EINVAL; }
    sp[i] = (uint8_t)(spc[i] - 1);
  }
  ASR_ON_DEVICE(ctx->device);
  asr_supercell* sc = new asr_supercell();
  sc->ctx = ctx; sc->n = nsite; sc->ns = nslot; sc->nsp = nsp;
  std::vector<int> nb((size_t)nslot * nsite);
  for (size_t q = 0; q < nb.size(); ++q) nb[q] = nbr[q] - 1;
  std::vector<double> par(4 * 9 * (size_t)nsp, 0.0);
  for (int q = 0; q < 9 * nsp; ++q) {
    par[q] = c[q];
    par[9 * nsp + q] = d[q];
    par[18 * nsp + q] = o ? o[q] : 0.0;
    par[27 * nsp + q] = e ? e[q] : 0.0;
    if (par[18 * nsp + q] != 0.0) sc->o_zero = false;
    if (par[27 * nsp + q] != 0.0) sc->e_zero = false;
  }
  std::vector<double> B((size_t)(nslot + 1) * 81, 0.0);
  for (int l = 0; l < 9; ++l)
    for (int lp = 0; lp < 9; ++lp) {
      if (block0) B[l * 9 + lp] = block0[l + 9 * lp];
      for (int k = 0; k < nslot; ++k) B[(size_t)(k + 1) * 81 + l * 9 + lp] = block[l + 9 * (lp + 9 * (size_t)k)];
    }
  std::vector<float> Bf(B.begin(), B.end());
  cudaStream_t s = ctx->stream;
  bool ok = cudaMalloc(&sc->d_nbr, std::max<size_t>(nb.size(), 1) * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&sc->d_spc, nsite) == cudaSuccess && cudaMalloc(&sc->d_par, par.size() * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&sc->d_blocks, B.size() * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&sc->d_blocks_f, Bf.size() * sizeof(float)) == cudaSuccess;
  if (!ok) { set_error("asr_supercell_build: device allocation failed"); delete sc; return ASR_ENOMEM; }
  cudaMemcpyAsync(sc->d_nbr, nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(sc->d_spc, sp.data(), nsite, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(sc->d_par, par.data(), par.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  sc->par_h = par;
  cudaMemcpyAsync(sc->d_blocks, B.data(), B.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(sc->d_blocks_f, Bf.data(), Bf.size() * sizeof(float), cudaMemcpyHostToDevice, s);
  ASR_CUDA(cudaStreamSynchronize(s));
  *out = sc;
  return ASR_OK;
}

int asr_supercell_free(asr_supercell* sc) {
  if (!sc) return ASR_OK;
  DeviceGuard dg;
  dg.set(sc->ctx->device);
  cudaFree(sc->d_nbr); cudaFree(sc->d_spc); cudaFree(sc->d_par); cudaFree(sc->d_blocks); cudaFree(sc->d_blocks_f);
  delete sc;
  return ASR_OK;
}

int asr_supercell_apply(asr_supercell* sc, const double* x, double* y, int nvec) {
  if (!sc || !x || !y || nvec < 1) { set_error("asr_supercell_apply: bad argument"); return ASR_EINVAL; }
  asr_ctx* ctx = sc->ctx;
  ASR_ON_DEVICE(ctx->device);
  cudaStream_t s = ctx->stream;
  const int n = sc->n;
  const size_t nel = (size_t)n * 9 * KV;
  ScView S{n, sc->ns, sc->nsp, sc->d_nbr, sc->d_spc, sc->d_par};
  const size_t smem = 4 * 9 * sc->nsp * sizeof(double) + (size_t)(sc->ns + 1) * 81 * sizeof(double);
  const int grid = ctx->num_sms * 4;
  for (int vb = 0; vb < nvec; vb += KV) {
    int nv = std::min(KV, nvec - vb);
    std::vector<double> hx(nel, 0.0), hy(nel);
    for (int v = 0; v < nv; ++v)
      for (size_t q = 0; q < (size_t)n * 9; ++q) hx[q * KV + v] = x[(size_t)(vb + v) * n * 9 + q];
    DevBuf<double> X, W1, W2, W3;
    ASR_TRY(X.alloc(nel)); ASR_TRY(W1.alloc(nel)); ASR_TRY(W2.alloc(nel)); ASR_TRY(W3.alloc(nel));
    ASR_CUDA(cudaMemcpyAsync(X.p, hx.data(), nel * sizeof(double), cudaMemcpyHostToDevice, s));
    k_h<double><<<grid, KSITES * KV, smem, s>>>(S, sc->d_blocks, X.p, false, W1.p);
    k_h<double><<<grid, KSITES * KV, smem, s>>>(S, sc->d_blocks, X.p, true, W2.p);   // o h x
    k_h<double><<<grid, KSITES * KV, smem, s>>>(S, sc->d_blocks, W2.p, false, W3.p);
    ASR_CUDA(cudaGetLastError());
    std::vector<double> w1(nel), w3(nel);
    ASR_CUDA(cudaMemcpyAsync(w1.data(), W1.p, nel * sizeof(double), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaMemcpyAsync(w3.data(), W3.p, nel * sizeof(double), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    // y = e x + h x - h o h x (real_apply, src/reference/asr_lmto_realization.f90:149-191)
    std::vector<double> par(4 * 9 * (size_t)sc->nsp);
    ASR_CUDA(cudaMemcpy(par.data(), sc->d_par, par.size() * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<uint8_t> sp(n);
    ASR_CUDA(cudaMemcpy(sp.data(), sc->d_spc, n, cudaMemcpyDeviceToHost));
    for (int v = 0; v < nv; ++v)
      for (int i = 0; i < n; ++i)
        for (int l = 0; l < 9; ++l) {
          size_t q = (size_t)i * 9 + l;
          double ev = par[27 * sc->nsp + l + 9 * sp[i]];
          y[(size_t)(vb + v) * n * 9 + q] = ev * x[(size_t)(vb + v) * n * 9 + q] + w1[q * KV + v] - w3[q * KV + v];
        }
  }
  return ASR_OK;
}

int asr_kpm_moments(asr_ctx* ctx, asr_supercell* sc, double cen, double scl, int nmom, int v0, int nvec, uint64_t seed,
                    int precision, int doubling, double* mu) {
  if (!ctx || !sc || !mu || nmom < 1 || nvec < 1 || !(scl > 0.0)) { set_error("kpm_moments: bad argument"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  if (precision == ASR_FP32) return kpm_run<float>(ctx, sc, cen, scl, nmom, v0, nvec, seed, doubling != 0, mu);
  return kpm_run<double>(ctx, sc, cen, scl, nmom, v0, nvec, seed, doubling != 0, mu);
}

// kpm_dos (src/reference/asr_kpm.f90:68-87): Jackson kernel, host
int asr_kpm_dos(const double* mu, int nmom, double cen, double scl, const double* e, int ne, double* rho) {
  if (!mu || !e || !rho || nmom < 1 || ne < 0 || !(scl > 0.0)) { set_error("kpm_dos: bad argument"); return ASR_EINVAL; }
  const double pi = 3.14159265358979323846;
  std::vector<double> g(nmom);
  for (int n = 0; n < nmom; ++n)
    g[n] = ((nmom - n + 1) * std::cos(pi * n / (nmom + 1)) + std::sin(pi * n / (nmom + 1)) / std::tan(pi / (nmom + 1))) / (nmom + 1);
  for (int i = 0; i < ne; ++i) {
    double x = (e[i] - cen) / scl;
    if (std::fabs(x) >= 1.0) { rho[i] = 0.0; continue; }
    double th = std::acos(x), s = g[0] * mu[0];
    for (int n = 1; n < nmom; ++n) s += 2.0 * g[n] * mu[n] * std::cos(n * th);
    rho[i] = s / (pi * std::sqrt(1.0 - x * x) * scl);
  }
  return ASR_OK;
}

}  // extern "C"
