// Batched Lanczos chains on the site-class operator (sm_100a).
//
// Reference: edc_green / edc_green_blk (src/asr_edc.f90:75-164, :237-316) with the block kernels of src/asr_augblk.f90
// (rand_r :88-124, rand_lin_amp :127-165, smul :170-203, hmul :206-215, blk_hamx :219-250, blk_project :284-304), and the
// plain real chain lanczos (src/reference/asr_recursion.f90:17-58) on augcls_apply (src/asr_augcls.f90:275-297).
//
// Layout: a tile holds TL = 32 chains ("lanes", one energy or one start vector each).  Every vector of a tile is stored
// node-major as x[((tile * nn + node) * 9 + orbital) * 32 + lane], so one warp covers one node of a tile and every
// load of a node's orbital is one 512-byte (FP64) or 256-byte (FP32) coalesced transaction.  The 9 x 9 bond blocks are
// kept unrotated in shared memory; the group operation of a link is applied to the gathered neighbour vector
// (orbital permutation pi(l, g) and signs chi(g) sg(l, g)), so the block table stays (1 + nslot) x 81 per site type
// instead of the reference's btab(9, 9, nslot, nop, ntype).
//
// One chain step (general operator H = E_nu + h - h o h, h = c + d S d, plus X(z) = z pa + pb) is a short sequence of
// node-parallel kernels; with d uniform and o = 0 (the edc route) it is one fused kernel: y = d S d x + (c + e + X(z)) x
// and the dot a = u . y.  Vectors are stored in amplitude coordinates (x = u / sqrt(orbit size)), so gathers need no
// scaling and the dots carry the orbit size; they are kept unnormalised with a complex scale per lane (x = s X); every
// kernel works on X and applies s once per node, which turns the normalisation u = w / b into a scalar update.  Tiles
// hold the lanes of one group, so d (folded into the shared-memory blocks) and the characters chi are per tile.
// Reductions (a, b) are per block partial sums in a fixed order followed by a per-tile pass, so the result is bitwise
// the same in every run.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "cf.cuh"
#include "chain.cuh"

namespace asrb {

namespace {

constexpr int WPB = 8;   // warps per block

__device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }

template <typename ST> struct St2;
template <> struct St2<double> { typedef double2 T; };
template <> struct St2<float> { typedef float2 T; };

__device__ __forceinline__ double2 ld(const double2* p) { return *p; }
__device__ __forceinline__ double2 ld(const float2* p) { float2 v = *p; return make_double2(v.x, v.y); }
__device__ __forceinline__ void stv(double2* p, double2 v) { *p = v; }
__device__ __forceinline__ void stv(float2* p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }
// evict-first store / last-use load: streams that are read once must not push the gathered vector out of L2
__device__ __forceinline__ void stv_cs(double2* p, double2 v) { __stcs(p, v); }
__device__ __forceinline__ void stv_cs(float2* p, double2 v) { __stcs(p, make_float2((float)v.x, (float)v.y)); }
__device__ __forceinline__ double2 ld_cs(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_cs(const float2* p) { float2 v = __ldcs(p); return make_double2(v.x, v.y); }

__device__ __forceinline__ size_t vix(int tile, int nn, int node, int l) {
  return (((size_t)tile * nn + node) * 9 + l) * TL;
}

// complex weight W_p + z W_pz (pz < 0: none) of the diagonal term for (l, own, flip) of class kap; the edc route's
// X(z) = z pa + pb enters as pz = PA
__device__ __forceinline__ double2 pweight(const double* gb, const GroupLayout& GL, int p, int pz, double2 z, int nsm,
                                           int kap, int own, int flip, int l) {
  int q = ((kap * nsm + own) * nsm + flip) * 9 + l;
  double w = p >= 0 ? __ldg(gb + GL.w(p) + q) : 0.0;
  if (pz >= 0) {
    double wa = __ldg(gb + GL.w(pz) + q);
    return make_double2(w + z.x * wa, z.y * wa);
  }
  return make_double2(w, 0.0);
}
__device__ __forceinline__ double2 praw(const double* gb, const GroupLayout& GL, int p, int pz, double2 z, int sp, int l) {
  int q = (sp - 1) * 9 + l;
  double w = p >= 0 ? __ldg(gb + GL.raw(p) + q) : 0.0;
  if (pz >= 0) {
    double wa = __ldg(gb + GL.raw(pz) + q);
    return make_double2(w + z.x * wa, z.y * wa);
  }
  return make_double2(w, 0.0);
}
__device__ __forceinline__ int frozen_of(const OpView& op, const GroupInfo& gi, int i) {
  return (op.start[i] && gi.frozen_sp > 0) ? gi.frozen_sp : (int)op.frozen[i];
}

// R_p(v) at node i for one lane: the random site-diagonal operator of apply_rand (src/asr_augcls.f90:380-403) on the
// vector v (unscaled, amplitude coordinates); xi_own: the node's own values of v.
template <typename T2>
__device__ __forceinline__ void rand_term(const OpView& op, const GroupInfo& gi, const double* gb, const GroupLayout& GL, int p,
                                          int pz, double2 z, const T2* v, int tile, int i, int lane, double2* out,
                                          const double2* xi_own) {
  int fs = frozen_of(op, gi, i);
  if (fs > 0) {
    for (int l = 0; l < 9; ++l) out[l] = cmul(praw(gb, GL, p, pz, z, fs, l), xi_own[l]);
    return;
  }
  const int nsm = op.nsmax;
  int kap = op.ncl[i], l0 = op.lst[i];
  for (int l = 0; l < 9; ++l) out[l] = cmul(pweight(gb, GL, p, pz, z, nsm, kap, l0, l0, l), xi_own[l]);
  int nk = op.nsc[kap];
  for (int k = 0; k < nk; ++k) {
    if (k == l0) continue;
    int r = op.flipr[k + nsm * i];
    if (r < 0) continue;
    int g = op.flipg[k + nsm * i];
    bool neg = (gi.chimask >> g) & 1ull;
    uint32_t sgm = op.sgm[g];
    for (int l = 0; l < 9; ++l) {
      int pl = op.pi[g * 9 + l];
      double2 x = ld(v + vix(tile, op.nn, r, pl) + lane);
      double sgn = (((sgm >> l) & 1u) ^ (neg ? 1u : 0u)) ? -1.0 : 1.0;
      out[l] = cadd(out[l], cmul(pweight(gb, GL, p, pz, z, nsm, kap, l0, k, l), cscale(x, sgn)));
    }
  }
}

struct NodeIter {   // nodes of a block: warp w of block-in-tile nb takes nb * npb + w + WPB * q, q < npw
  int tile, first, npw, nn;
};
__device__ __forceinline__ bool node_iter(const BatchView& bv, int npw, NodeIter& it, int& bpt) {
  int npb = WPB * npw;
  bpt = (bv.nn + npb - 1) / npb;
  int b = blockIdx.x;
  it.tile = b / bpt;
  it.first = (b % bpt) * npb;
  it.npw = npw;
  it.nn = bv.nn;
  return it.tile < bv.ntile && bv.tile_act[it.tile];
}

// block-level fixed-order reduction of one double2 per lane over the warps; writes part[(tile * bpt + nb) * TL + lane]
__device__ __forceinline__ void block_reduce_store(double2 v, double2* part, int tile, int bpt) {
  __shared__ double2 red[WPB][TL];
  int w = threadIdx.x / TL, lane = threadIdx.x % TL;
  red[w][lane] = v;
  __syncthreads();
  if (w == 0) {
    double2 s = red[0][lane];
    for (int q = 1; q < WPB; ++q) s = cadd(s, red[q][lane]);
    part[((size_t)tile * bpt + blockIdx.x % bpt) * TL + lane] = s;
  }
}

// sum_{q < n} p[q * stride] (one double2 per lane, p[lane] the first row) over the warps of the calling block (every
// thread calls it; at most WPB warps): warp w adds the rows q = w, w + nw, ... in order with the loads issued eight at
// a time (one L2 latency per eight rows of the nn / 32 partials of a tile), then warp 0 adds the nw warp sums in the
// order w = 0 .. nw - 1.
// A fixed order, so the same bits on every run; the result is valid in warp 0 (lane = threadIdx.x).
__device__ __forceinline__ double2 block_sum_rows(const double2* __restrict__ p, int n, size_t stride, bool load = true) {
  __shared__ double2 wsum[WPB][TL];
  const int nw = blockDim.x / TL, w = threadIdx.x / TL, lane = threadIdx.x % TL;
  const double2* pl = p + lane;
  double2 s = make_double2(0, 0);
  int q = load ? w : n;   // a lane without a column (load = false) adds nothing
  for (; q + 7 * nw < n; q += 8 * nw) {
    double2 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = __ldcg(pl + (size_t)(q + j * nw) * stride);
#pragma unroll
    for (int j = 0; j < 8; ++j) s = cadd(s, v[j]);
  }
  for (; q < n; q += nw) s = cadd(s, __ldcg(pl + (size_t)q * stride));
  wsum[w][lane] = s;
  __syncthreads();
  if (w == 0)
    for (int k = 1; k < nw; ++k) s = cadd(s, wsum[k][lane]);
  __syncthreads();
  return s;
}

// Ticket of a finished block: true in every thread of the block of `tile` that stored its partials last, once all bpt
// blocks of the tile have stored theirs (no block waits on another).  The last block resets the ticket for the next
// launch.  Every thread of the block calls it, after block_reduce_store.
__device__ __forceinline__ bool last_block_of_tile(int* tick, int tile, int bpt) {
  __shared__ int s_last;
  __threadfence();   // the partials this block stored, before its ticket
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(tick + tile, 1);
    s_last = t == bpt - 1;
    if (s_last) tick[tile] = 0;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last != 0;
}

// a_k (asum: the tile's partials summed by block_sum_rows) for one lane of a tile; depth test every 4 levels from 8
// (src/asr_edc.f90:121-127) when DEPTH (without it the caller guarantees that no depth test is due at level k)
template <bool DEPTH>
__device__ __forceinline__ void reduce_a_lane(const BatchView& bv, double2 asum, int k, int tile, int lane) {
  int L = tile * TL + lane;
  int grp = bv.lane_group[L];
  bv.lane_wact[L] = 0;
  if (grp < 0 || !bv.lane_act[L]) return;
  const double2 a = asum;
  bv.acur[L] = a;
  bv.acoef[(size_t)L * NLMAX + k - 1] = a;
  bv.lane_m[L] = k;
  int nlev = bv.ginfo[grp].nlev;
  bool go = true;
  if (k == nlev) {
    go = false;   // edc exits before b_k (src/asr_edc.f90:120); the plain chain still forms b_n (asr_recursion.f90:50-57)
    if (bv.mode == ASR_MODE_PLAIN) bv.lane_wact[L] = 1;
  } else if (DEPTH && bv.depth_tol > 0.0 && k >= 8 && k % 4 == 0 && bv.mode == ASR_MODE_EDC) {
    double2 wd[NLMAX], we[NLMAX];
    int nf = 0;
    double2 gtry = cf_species_dev(bv.acoef + (size_t)L * NLMAX, bv.bcoef + (size_t)L * NLMAX, k, bv.lane_z[L], bv.tail, wd, we,
                                  &nf, nullptr);
    if (nf) atomicAdd(bv.nfall, nf);
    if (k > 8 && cmag(csub(gtry, bv.gprev[L])) <= bv.depth_tol * cmag(gtry)) go = false;   // :123-125
    bv.gprev[L] = gtry;
  }
  if (go) bv.lane_wact[L] = 1;
  else bv.lane_act[L] = 0;
}

// b_k = sqrt(w . w) (wsum: the tile's partials summed by block_sum_rows); |b| < tol ends the chain; scales of the next
// step (u <- w / b, up <- u).  One full warp per tile.
__device__ __forceinline__ void reduce_b_lane(const BatchView& bv, double2 wsum, int k, double btol, int tile, int lane,
                                              bool tile_live) {
  int L = tile * TL + lane;
  int grp = bv.lane_group[L];
  bool act = false;
  if (tile_live && grp >= 0 && bv.lane_wact[L]) {
    const double2 ww = wsum;
    double2 b = bv.mode == ASR_MODE_PLAIN ? make_double2(sqrt(ww.x), 0.0) : csqrt_p(ww);
    bv.bcoef[(size_t)L * NLMAX + k - 1] = b;
    bool ok = bv.mode == ASR_MODE_PLAIN ? (b.x >= btol) : (cmag(b) >= btol);   // |b| < 1e-12 ends the chain
    if (!bv.lane_act[L]) ok = false;   // plain chain at its last level: b_n stored, chain done
    else if (!ok && bv.lane_closed) bv.lane_closed[L] = 1;   // the Krylov space is exhausted
    if (ok) {
      bv.sup[L] = bv.su[L];
      bv.su[L] = cdiv(make_double2(1.0, 0.0), b);
      bv.bprev[L] = b;
      act = true;
    } else {
      bv.lane_act[L] = 0;
    }
  }
  if (!act) {
    bv.su[L] = make_double2(0, 0);
    bv.sup[L] = make_double2(0, 0);
  }
  // tile activity for the next step (a warp vote over the lanes)
  unsigned any = __ballot_sync(0xffffffffu, act);
  if (lane == 0) bv.tile_act[tile] = any != 0;
}

// sign flip of a complex value by the sign bit (no floating-point operation)
__device__ __forceinline__ double2 flip_if(double2 x, uint32_t bit) {
  unsigned long long m = (unsigned long long)bit << 63;
  return make_double2(__longlong_as_double(__double_as_longlong(x.x) ^ m), __longlong_as_double(__double_as_longlong(x.y) ^ m));
}
__device__ __forceinline__ float2 flip_if(float2 x, uint32_t bit) {
  unsigned m = bit << 31;
  return make_float2(__uint_as_float(__float_as_uint(x.x) ^ m), __uint_as_float(__float_as_uint(x.y) ^ m));
}
template <typename ST> struct Pair;
template <> struct Pair<double> { typedef double2 T; };
template <> struct Pair<float> { typedef float2 T; };

constexpr int RW = 12;   // padded row of a shared-memory block (16-byte aligned pairs for FP64 and FP32)

// Block products of the step kernel: acc_l += sum_lp B[l][lp] x[lp] over the nine rows of one shared-memory block, the
// nine products of a row added in the order lp = 0 .. 8.  FP64: rows of RW doubles.  FP32: rows 2p and 2p + 1 (p < 4)
// interleaved as {B[2p][lp], B[2p+1][lp]} pairs (18 floats, padded to 20), then row 8 alone (padded to 12); one paired
// FMA (__ffma2_rn, each half rounded as a scalar FMA) updates one component of two rows, so the bits are those of the
// scalar products with half their FMA instructions and no more shared-memory bytes.
template <typename ST> struct BlockAcc;
template <> struct BlockAcc<double> {
  static constexpr int BLK = 9 * RW;   // elements per block
  __device__ static void put(double* blk, int l, int lp, double v) { blk[l * RW + lp] = v; }
  double2 a[9];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int l = 0; l < 9; ++l) a[l] = make_double2(0.0, 0.0);
  }
  __device__ __forceinline__ void mac(const double* __restrict__ blk, const double2* x) {
#pragma unroll
    for (int l = 0; l < 9; ++l) {
      const double* row = blk + l * RW;
#pragma unroll
      for (int lp = 0; lp < 8; lp += 2) {
        const double2 bb = *(const double2*)(row + lp);
        a[l].x = fma(bb.x, x[lp].x, a[l].x);
        a[l].y = fma(bb.x, x[lp].y, a[l].y);
        a[l].x = fma(bb.y, x[lp + 1].x, a[l].x);
        a[l].y = fma(bb.y, x[lp + 1].y, a[l].y);
      }
      a[l].x = fma(row[8], x[8].x, a[l].x);
      a[l].y = fma(row[8], x[8].y, a[l].y);
    }
  }
  __device__ __forceinline__ void out(double2* acc) const {
#pragma unroll
    for (int l = 0; l < 9; ++l) acc[l] = a[l];
  }
};
template <> struct BlockAcc<float> {
  static constexpr int BLK = 4 * 20 + 12;
  __device__ static void put(float* blk, int l, int lp, double v) {
    if (l < 8) blk[(l >> 1) * 20 + 2 * lp + (l & 1)] = (float)v;
    else blk[80 + lp] = (float)v;
  }
  float2 ax[4], ay[4], a8;   // {row 2p, row 2p + 1} of the real and of the imaginary parts; row 8
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int p = 0; p < 4; ++p) { ax[p] = make_float2(0.f, 0.f); ay[p] = ax[p]; }
    a8 = make_float2(0.f, 0.f);
  }
  __device__ __forceinline__ void mac(const float* __restrict__ blk, const float2* x) {
#pragma unroll
    for (int lp = 0; lp < 8; lp += 2) {
      const float2 x0 = make_float2(x[lp].x, x[lp].x), y0 = make_float2(x[lp].y, x[lp].y);
      const float2 x1 = make_float2(x[lp + 1].x, x[lp + 1].x), y1 = make_float2(x[lp + 1].y, x[lp + 1].y);
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const float4 bb = *(const float4*)(blk + p * 20 + 2 * lp);
        ax[p] = __ffma2_rn(make_float2(bb.x, bb.y), x0, ax[p]);
        ay[p] = __ffma2_rn(make_float2(bb.x, bb.y), y0, ay[p]);
        ax[p] = __ffma2_rn(make_float2(bb.z, bb.w), x1, ax[p]);
        ay[p] = __ffma2_rn(make_float2(bb.z, bb.w), y1, ay[p]);
      }
    }
    {
      const float2 x8 = make_float2(x[8].x, x[8].x), y8 = make_float2(x[8].y, x[8].y);
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const float2 bb = *(const float2*)(blk + p * 20 + 16);
        ax[p] = __ffma2_rn(bb, x8, ax[p]);
        ay[p] = __ffma2_rn(bb, y8, ay[p]);
      }
    }
    const float* r8 = blk + 80;
#pragma unroll
    for (int lp = 0; lp < 8; lp += 2) {
      const float2 bb = *(const float2*)(r8 + lp);
      a8.x = fmaf(bb.x, x[lp].x, a8.x);
      a8.y = fmaf(bb.x, x[lp].y, a8.y);
      a8.x = fmaf(bb.y, x[lp + 1].x, a8.x);
      a8.y = fmaf(bb.y, x[lp + 1].y, a8.y);
    }
    a8.x = fmaf(r8[8], x[8].x, a8.x);
    a8.y = fmaf(r8[8], x[8].y, a8.y);
  }
  __device__ __forceinline__ void out(float2* acc) const {
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      acc[2 * p] = make_float2(ax[p].x, ay[p].x);
      acc[2 * p + 1] = make_float2(ax[p].y, ay[p].y);
    }
    acc[8] = a8;
  }
};

// packed orbital operation of the identity: permutation pi(l) = l in bits 4l..4l+3, no signs (bits 40..48)
constexpr unsigned long long PW_IDENTITY = 0x876543210ull;
constexpr unsigned long long PW_PERM_MASK = 0xFFFFFFFFFull;   // the nine 4-bit orbital indices

// the output of one node of the S application: t2 (unscaled), or with FINAL y = s (d t2 + (c + e + X(z)) U) and the
// node's share of the dot sum norb (s U) . y.  EPI 1: also t2 = S (d o U) into bv.t2out.  EPI 2 (the adjoint, U = wbar_k,
// unit scales): t2 into bv.t2out and, in place of y, ubar_k = y + ca Y_k - cb U - cc wbar_{k+1} into bv.adj.ubk, the dot
// being sum norb ubar_k . X_k (raw)
template <typename ST, bool FINAL, int EPI = 0, typename T2, typename A2>
__device__ __forceinline__ void smul_node_out(const OpView& op, const BatchView& bv, int tile, int i, int lane, int L, int grp,
                                              int gflags, int gfrozen, const unsigned long long* piw, const T2* __restrict__ in,
                                              T2* __restrict__ out, const A2* acc, double2& dot) {
  if (!FINAL) {
#pragma unroll
    for (int l = 0; l < 9; ++l) stv(out + vix(tile, bv.nn, i, l) + lane, make_double2(acc[l].x, acc[l].y));
  } else {
    // y_l = s (d_l t2_l + P_l(U)),  P = c + e + X(z) (src/asr_augblk.f90:219-250), orbital by orbital
    const double* gb = bv.gblob + (size_t)(grp >= 0 ? grp : 0) * bv.GL.stride;
    const double2 z = bv.lane_z[L];
    const double2 s = bv.su[L];
    const bool withx = !(gflags & GF_X_ZERO);
    const double norb = op.sq[i] * op.sq[i];
    const int fs = (op.start[i] && gfrozen > 0) ? gfrozen : (int)op.frozen[i];
    const int nsm = op.nsmax, kap = op.ncl[i], l0 = op.lst[i], nk = op.nsc[kap];
    double2 ea = make_double2(0, 0), eb = ea, ec = ea;
    if (EPI == 2) { ea = bv.adj.ca[L]; eb = bv.adj.cb[L]; ec = bv.adj.cc[L]; }
#pragma unroll
    for (int l = 0; l < 9; ++l) {
      double2 ui = ld(in + vix(tile, bv.nn, i, l) + lane);
      double2 pt;
      if (fs > 0) {
        pt = cmul(praw(gb, bv.GL, PCEB, withx ? PA : -1, z, fs, l), ui);
      } else {
        pt = cmul(pweight(gb, bv.GL, PCEB, withx ? PA : -1, z, nsm, kap, l0, l0, l), ui);
        for (int k = 0; k < nk; ++k) {
          if (k == l0) continue;
          int r = op.flipr[k + nsm * i];
          if (r < 0) continue;
          const unsigned long long pw = piw[op.flipg[k + nsm * i]];
          int p = (int)((pw >> (4 * l)) & 15ull);
          double2 xr = flip_if(ld(in + vix(tile, bv.nn, r, p) + lane), (uint32_t)((pw >> (40 + l)) & 1ull));
          pt = cadd(pt, cmul(pweight(gb, bv.GL, PCEB, withx ? PA : -1, z, nsm, kap, l0, k, l), xr));
        }
      }
      double2 y = cmul(s, cadd(make_double2(acc[l].x, acc[l].y), pt));
      const size_t q = vix(tile, bv.nn, i, l) + lane;
      if (EPI != 2) stv_cs(out + q, y);
      if (EPI >= 1) {   // the blocks carry d on both sides: t2 = S (d o U) = acc / d_l
        const double il = 1.0 / bv.ginfo[grp >= 0 ? grp : 0].dd[l];
        stv((T2*)bv.t2out + q, make_double2(acc[l].x * il, acc[l].y * il));
      }
      if (EPI == 2) {
        double2 ub = cadd(y, cmul(ea, ld((const T2*)bv.adj.yk + q)));
        ub = csub(ub, cmul(eb, ui));
        ub = csub(ub, cmul(ec, ld((const T2*)bv.adj.wbn + q)));
        stv((T2*)bv.adj.ubk + q, ub);
        dot = cadd(dot, cscale(cmul(ub, ld((const T2*)bv.adj.xk + q)), norb));
      } else {
        dot = cadd(dot, cscale(cmul(cmul(s, ui), y), norb));
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------ S application
// t2 = S t1 (src/asr_augcls.f90:456-477 / src/asr_augblk.f90:170-203), unscaled amplitude coordinates.
// FUSE_D: t1 = d o U is folded into the shared-memory blocks (the tile's d per orbital; d is invariant under the orbital
// permutations of the group).  FINAL (needs FUSE_D, o = 0): y = s (d o S d o U + (c + e + X(z)) U) and the partial dot
// sum_i norb_i (s U_i) . y_i (normalised-coordinate bilinear form).  Group data are per tile (single-group tiles).
// LINK_ID: links whose orbital operation keeps the orbital order (the identity, and the pure sign changes of diagonal
// groups such as D2h) gather their nine rows at fixed offsets, without the per-orbital index and sign decoding; the
// products and their order are those of the general path, so both instantiations give the same bits.
template <typename ST, bool FUSE_D, bool FINAL, bool LINK_ID, int EPI = 0>
__global__ void __launch_bounds__(WPB * TL) k_smul(OpView op, BatchView bv, const ST* __restrict__ blocks,
                                                   const typename St2<ST>::T* __restrict__ in,
                                                   typename St2<ST>::T* __restrict__ out, double2* part, int npw) {
  typedef typename St2<ST>::T T2;
  typedef typename Pair<ST>::T P2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ns1 = op.nslot + 1;
  ST* Bs = (ST*)smem_raw;                                                        // [ntype][ns1][9][RW]
  unsigned long long* piw = (unsigned long long*)(smem_raw + (((size_t)op.ntype * ns1 * BlockAcc<ST>::BLK * sizeof(ST) + 15) & ~(size_t)15));
  NodeIter it;
  int bpt;
  bool live = node_iter(bv, npw, it, bpt);
  const int grp = live ? bv.tile_group[it.tile] : -1;
  unsigned long long chimask = 0ull;
  int gflags = 0, gfrozen = 0;
  if (grp >= 0) {
    chimask = bv.ginfo[grp].chimask;
    gflags = bv.ginfo[grp].flags;
    gfrozen = bv.ginfo[grp].frozen_sp;
  }
  {
    const double* dd = grp >= 0 ? bv.ginfo[grp].dd : nullptr;
    const int nb = op.ntype * ns1 * 81;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
      int lp = q % 9, l = (q / 9) % 9, tk = q / 81;
      double v = (double)blocks[q];
      if (FUSE_D && dd) v *= dd[lp];
      if (FINAL && dd) v *= dd[l];
      BlockAcc<ST>::put(Bs + (size_t)tk * BlockAcc<ST>::BLK, l, lp, v);
    }
    for (int g = threadIdx.x; g < op.nop; g += blockDim.x) {
      unsigned long long w = 0ull;
      for (int l = 0; l < 9; ++l) w |= (unsigned long long)op.pi[g * 9 + l] << (4 * l);
      uint32_t sg = op.sgm[g] ^ (((chimask >> g) & 1ull) ? 0x1FFu : 0u);
      piw[g] = w | ((unsigned long long)sg << 40);
    }
  }
  __syncthreads();
  if (!live) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  double2 dot = make_double2(0.0, 0.0);
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    const ST* B = Bs + (size_t)op.typ[i] * ns1 * BlockAcc<ST>::BLK;
    BlockAcc<ST> A;
    A.zero();
    {   // on-site block
      const T2* src = in + vix(it.tile, bv.nn, i, 0) + lane;
      T2 v[9];
      for (int l2 = 0; l2 < 9; ++l2) v[l2] = src[l2 * TL];
      A.mac(B, v);
    }
    // the node's links, one slot per lane, read once with a coalesced load and broadcast by shuffles: the row gathers
    // then wait on one global latency per slot instead of two dependent ones (link, then row)
    const bool lane_links = op.nslot <= TL;
    int my_r = -1, my_g = 0;
    if (lane_links && lane < op.nslot) { my_r = op.hopr[lane + op.nslot * i]; my_g = op.hopg[lane + op.nslot * i]; }
    for (int k = 0; k < op.nslot; ++k) {
      int r, gk;
      if (lane_links) {
        r = __shfl_sync(0xffffffffu, my_r, k);
        gk = __shfl_sync(0xffffffffu, my_g, k);
      } else {
        r = op.hopr[k + op.nslot * i];
        gk = op.hopg[k + op.nslot * i];
      }
      if (r < 0) continue;
      const unsigned long long pw = piw[gk];
      const T2* src = in + vix(it.tile, bv.nn, r, 0) + lane;
      T2 v[9];
      if (LINK_ID && pw == PW_IDENTITY) {                                        // warp-uniform: one node, one slot
        for (int lp = 0; lp < 9; ++lp) v[lp] = src[lp * TL];
      } else if (LINK_ID && (pw & PW_PERM_MASK) == PW_IDENTITY) {               // signs only
        const uint32_t sg = (uint32_t)(pw >> 40);
        for (int lp = 0; lp < 9; ++lp) v[lp] = flip_if(src[lp * TL], (sg >> lp) & 1u);
      } else {
        for (int lp = 0; lp < 9; ++lp) {
          int p = (int)((pw >> (4 * lp)) & 15ull);
          v[lp] = flip_if(src[p * TL], (uint32_t)((pw >> (40 + lp)) & 1ull));
        }
      }
      A.mac(B + (size_t)(k + 1) * BlockAcc<ST>::BLK, v);
    }
    T2 acc[9];
    A.out(acc);
    smul_node_out<ST, FINAL, EPI>(op, bv, it.tile, i, lane, L, grp, gflags, gfrozen, piw, in, out, acc, dot);
  }
  if (FINAL) {
    block_reduce_store(dot, part, it.tile, bpt);
    if (bv.tick && last_block_of_tile(bv.tick, it.tile, bpt)) {
      const double2 a = block_sum_rows(part + (size_t)it.tile * bpt * TL, bpt, TL);
      if (threadIdx.x < TL) reduce_a_lane<false>(bv, a, bv.kstep, it.tile, threadIdx.x);
    }
  }
}

// ------------------------------------------------------------------------------------------------ staged S application
// The same product with the neighbour rows staged in shared memory by the bulk-copy engine: one node's nine rows of a
// tile are contiguous (9 x 32 lanes), so lane 0 of each warp copies whole rows with cp.async.bulk into a ring of NST
// stages per warp, completion counted on one mbarrier per stage, while the warp multiplies the previous rows out of
// shared memory.  The gathers then cost no registers and no load latency in the FMA stream.  Every wait is bounded: on
// timeout the warp records an error, stops computing, drains its copies (bounded) and still reaches the block barrier.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* mb, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mb)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mb, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mb)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mb) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(mb))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mb, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(mb)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

constexpr int SMUL_NST = 2;            // stages per warp
constexpr long SMUL_WAIT_LIMIT = 1L << 24;

size_t smul_smem(const asr_op* op, size_t st_size);

template <typename ST>
size_t smul_bulk_smem(const asr_op* op) {
  typedef typename St2<ST>::T T2;
  size_t b = smul_smem(op, sizeof(ST));
  b = (b + 127) & ~(size_t)127;
  b += (size_t)WPB * SMUL_NST * 9 * TL * sizeof(T2);
  b += (size_t)WPB * SMUL_NST * sizeof(uint64_t);
  return b;
}

// acc += B x with x the staged rows (row pi(lp) for column lp, signs of pw)
template <typename ST, typename T2>
__device__ __forceinline__ void mac9_staged(const ST* __restrict__ Bk, const T2* __restrict__ rows, unsigned long long pw, T2* acc) {
  typedef typename Pair<ST>::T P2;
  T2 x[9];
#pragma unroll
  for (int lp = 0; lp < 9; ++lp)
    x[lp] = flip_if(rows[(int)((pw >> (4 * lp)) & 15ull) * TL], (uint32_t)((pw >> (40 + lp)) & 1ull));
#pragma unroll
  for (int l = 0; l < 9; ++l) {
    const ST* row = Bk + l * RW;
#pragma unroll
    for (int lp = 0; lp < 8; lp += 2) {
      P2 bb = *(const P2*)(row + lp);
      acc[l].x = fma_(bb.x, x[lp].x, acc[l].x);
      acc[l].y = fma_(bb.x, x[lp].y, acc[l].y);
      acc[l].x = fma_(bb.y, x[lp + 1].x, acc[l].x);
      acc[l].y = fma_(bb.y, x[lp + 1].y, acc[l].y);
    }
    acc[l].x = fma_(row[8], x[8].x, acc[l].x);
    acc[l].y = fma_(row[8], x[8].y, acc[l].y);
  }
}

template <typename ST, bool FUSE_D, bool FINAL>
__global__ void __launch_bounds__(WPB * TL) k_smul_bulk(OpView op, BatchView bv, const ST* __restrict__ blocks,
                                                        const typename St2<ST>::T* __restrict__ in,
                                                        typename St2<ST>::T* __restrict__ out, double2* part, int npw, int* err) {
  typedef typename St2<ST>::T T2;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int ns1 = op.nslot + 1;
  ST* Bs = (ST*)smem_raw;                                                        // [ntype][ns1][9][RW]
  const size_t bs_bytes = ((size_t)op.ntype * ns1 * 9 * RW * sizeof(ST) + 15) & ~(size_t)15;
  unsigned long long* piw = (unsigned long long*)(smem_raw + bs_bytes);
  const size_t stage_off = (bs_bytes + (size_t)op.nop * sizeof(unsigned long long) + 127) & ~(size_t)127;
  T2* stages = (T2*)(smem_raw + stage_off);                                     // [WPB][NST][9][TL]
  uint64_t* mbar = (uint64_t*)(smem_raw + stage_off + (size_t)WPB * SMUL_NST * 9 * TL * sizeof(T2));
  NodeIter it;
  int bpt;
  bool live = node_iter(bv, npw, it, bpt);
  const int grp = live ? bv.tile_group[it.tile] : -1;
  unsigned long long chimask = 0ull;
  int gflags = 0, gfrozen = 0;
  if (grp >= 0) {
    chimask = bv.ginfo[grp].chimask;
    gflags = bv.ginfo[grp].flags;
    gfrozen = bv.ginfo[grp].frozen_sp;
  }
  {
    const double* dd = grp >= 0 ? bv.ginfo[grp].dd : nullptr;
    const int nb = op.ntype * ns1 * 81;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
      int lp = q % 9, l = (q / 9) % 9, tk = q / 81;
      double v = (double)blocks[q];
      if (FUSE_D && dd) v *= dd[lp];
      if (FINAL && dd) v *= dd[l];
      Bs[((size_t)tk * 9 + l) * RW + lp] = (ST)v;
    }
    for (int g = threadIdx.x; g < op.nop; g += blockDim.x) {
      unsigned long long w = 0ull;
      for (int l = 0; l < 9; ++l) w |= (unsigned long long)op.pi[g * 9 + l] << (4 * l);
      uint32_t sg = op.sgm[g] ^ (((chimask >> g) & 1ull) ? 0x1FFu : 0u);
      piw[g] = w | ((unsigned long long)sg << 40);
    }
    if (threadIdx.x < WPB * SMUL_NST) mbar_init(mbar + threadIdx.x, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (!live) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  T2* stg = stages + (size_t)w * SMUL_NST * 9 * TL;
  uint64_t* mb = mbar + w * SMUL_NST;
  const uint32_t slab = 9 * TL * sizeof(T2);
  double2 dot = make_double2(0.0, 0.0);
  // slab stream of this warp: for each of its nodes, the own rows (slot -1) then every slot with a neighbour
  auto node_of = [&](int qn) { return it.first + w + WPB * qn; };
  auto valid_node = [&](int qn) { return qn < npw && node_of(qn) < bv.nn; };
  auto next_slot = [&](int i, int k) {   // next slot after k with a neighbour, nslot if none
    int kk = k + 1;
    while (kk < op.nslot && op.hopr[kk + op.nslot * i] < 0) ++kk;
    return kk;
  };
  int pq = 0, pk = -1;          // producer position
  bool pdone = !valid_node(0);
  auto issue = [&](int s) {     // lane 0: copy the producer's slab into stage s, then advance the producer
    const int i = node_of(pq);
    const int r = pk < 0 ? i : op.hopr[pk + op.nslot * i];
    if (lane == 0) {
      mbar_expect_tx(mb + s, slab);
      bulk_g2s(stg + (size_t)s * 9 * TL, in + vix(it.tile, bv.nn, r, 0), slab, mb + s);
    }
    pk = next_slot(i, pk);
    if (pk >= op.nslot) { ++pq; pk = -1; pdone = !valid_node(pq); }
  };
  for (int s = 0; s < SMUL_NST && !pdone; ++s) issue(s);
  bool ok = true;
  long t = 0;
  int cq = 0, ck = -1;
  bool cdone = !valid_node(0);
  T2 acc[9];
  for (int l = 0; l < 9; ++l) { acc[l].x = 0; acc[l].y = 0; }
  while (!cdone) {
    const int s = (int)(t % SMUL_NST);
    const uint32_t parity = (uint32_t)((t / SMUL_NST) & 1);
    if (ok) {
      long n = 0;
      while (!mbar_try_wait(mb + s, parity)) {
        if (++n > SMUL_WAIT_LIMIT) { ok = false; if (lane == 0) dev_fail(err, DERR_WAIT); break; }
      }
    }
    const int i = node_of(cq);
    if (ok) {
      const ST* B = Bs + (size_t)op.typ[i] * ns1 * 9 * RW;
      const unsigned long long pw = ck < 0 ? PW_IDENTITY : piw[op.hopg[ck + op.nslot * i]];
      mac9_staged<ST>(B + (size_t)(ck + 1) * 9 * RW, stg + (size_t)s * 9 * TL + lane, pw, acc);
    }
    __syncwarp();
    if (ok && !pdone) {
      if (lane == 0) fence_proxy_async_smem();
      issue(s);
    }
    ++t;
    ck = next_slot(i, ck);
    if (ck >= op.nslot) {   // the node is complete
      if (ok) smul_node_out<ST, FINAL>(op, bv, it.tile, i, lane, L, grp, gflags, gfrozen, piw, in, out, acc, dot);
      for (int l = 0; l < 9; ++l) { acc[l].x = 0; acc[l].y = 0; }
      ++cq;
      ck = -1;
      cdone = !valid_node(cq);
    }
  }
  if (!ok) {   // drain: the copies issued after the failed wait (bounded)
    for (int s = 0; s < SMUL_NST; ++s) {
      long n = 0;
      while (!mbar_try_wait(mb + s, (uint32_t)(((t + s) / SMUL_NST) & 1)) && ++n < SMUL_WAIT_LIMIT) {}
    }
  }
  if (FINAL) block_reduce_store(dot, part, it.tile, bpt);
}

// ------------------------------------------------------------------------------------------------ random operators
// out = R_p(in), amplitude coordinates, unscaled
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_rand(OpView op, BatchView bv, int p, const typename St2<ST>::T* __restrict__ in,
                                                   typename St2<ST>::T* __restrict__ out, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = bv.lane_group[L];
  if (grp < 0) return;
  const GroupInfo gi = bv.ginfo[grp];
  const double* gb = bv.gblob + (size_t)grp * bv.GL.stride;
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    double2 xi[9], o[9];
    for (int l = 0; l < 9; ++l) xi[l] = ld(in + vix(it.tile, bv.nn, i, l) + lane);
    rand_term(op, gi, gb, bv.GL, p, -1, make_double2(0, 0), in, it.tile, i, lane, o, xi);
    for (int l = 0; l < 9; ++l) stv(out + vix(it.tile, bv.nn, i, l) + lane, o[l]);
  }
}

// out = sgnAB (A + B) + C + H, A = D t2 (uniform: d o t2), B = R_pB(v1) (+ z pa if bx), C = R_(e+pb) + z pa on U
// (optional), H = h1 (optional), amplitude coordinates.  final: y = s out and the partial dot sum norb (s U) . y; else
// out is written unscaled.
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_combine(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ t2,
                                                      const typename St2<ST>::T* __restrict__ v1, int pB, bool bx,
                                                      const typename St2<ST>::T* __restrict__ u, bool cterm,
                                                      const typename St2<ST>::T* __restrict__ h1, double sgnAB, bool final_,
                                                      typename St2<ST>::T* __restrict__ out, double2* part, int npw) {
  NodeIter it;
  int bpt;
  bool live = node_iter(bv, npw, it, bpt);
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  double2 dot = make_double2(0.0, 0.0);
  if (live) {
    const int L = it.tile * TL + lane;
    const int grp = bv.lane_group[L];
    if (grp >= 0) {
      const GroupInfo gi = bv.ginfo[grp];
      const double* gb = bv.gblob + (size_t)grp * bv.GL.stride;
      const double2 z = bv.lane_z[L];
      const double2 s = bv.su[L];
      for (int qn = 0; qn < npw; ++qn) {
        int i = it.first + w + WPB * qn;
        if (i >= bv.nn) break;
        double2 acc[9], tmp[9], xi[9];
        if (t2) {
          for (int l = 0; l < 9; ++l) xi[l] = ld(t2 + vix(it.tile, bv.nn, i, l) + lane);
          if (gi.flags & GF_D_UNIFORM) for (int l = 0; l < 9; ++l) acc[l] = cscale(xi[l], gi.dd[l]);
          else rand_term(op, gi, gb, bv.GL, PD, -1, z, t2, it.tile, i, lane, acc, xi);
        } else {
          for (int l = 0; l < 9; ++l) acc[l] = make_double2(0, 0);
        }
        if (v1) {
          for (int l = 0; l < 9; ++l) xi[l] = ld(v1 + vix(it.tile, bv.nn, i, l) + lane);
          rand_term(op, gi, gb, bv.GL, pB, bx ? PA : -1, z, v1, it.tile, i, lane, tmp, xi);
          for (int l = 0; l < 9; ++l) acc[l] = cadd(acc[l], tmp[l]);
        }
        for (int l = 0; l < 9; ++l) acc[l] = cscale(acc[l], sgnAB);
        double2 ui[9];
        for (int l = 0; l < 9; ++l) ui[l] = ld(u + vix(it.tile, bv.nn, i, l) + lane);
        if (cterm) {
          rand_term(op, gi, gb, bv.GL, PEB, (gi.flags & GF_X_ZERO) ? -1 : PA, z, u, it.tile, i, lane, tmp, ui);
          for (int l = 0; l < 9; ++l) acc[l] = cadd(acc[l], tmp[l]);
        }
        if (h1) for (int l = 0; l < 9; ++l) acc[l] = cadd(acc[l], ld(h1 + vix(it.tile, bv.nn, i, l) + lane));
        if (final_) {
          const double norb = op.sq[i] * op.sq[i];
          for (int l = 0; l < 9; ++l) {
            double2 y = cmul(s, acc[l]);
            stv(out + vix(it.tile, bv.nn, i, l) + lane, y);
            dot = cadd(dot, cscale(cmul(cmul(s, ui[l]), y), norb));
          }
        } else {
          for (int l = 0; l < 9; ++l) stv(out + vix(it.tile, bv.nn, i, l) + lane, acc[l]);
        }
      }
    }
  }
  if (final_ && live) block_reduce_store(dot, part, it.tile, bpt);
}

// ------------------------------------------------------------------------------------------------ Lanczos update
// w = y - a u - b up (u = su U, up = sup UP); projection onto the symmetric subspace (augcls_project_c,
// src/asr_augcls.f90:329-348; node-local, the same in amplitude coordinates); lanes that left the chain are zeroed.
// w overwrites y; partial dot sum norb w . w.
__device__ __forceinline__ void project_node(const OpView& op, int i, unsigned long long chimask, double2* x) {
  int s0 = op.stab_ptr[i], s1 = op.stab_ptr[i + 1];
  int ns = s1 - s0;
  if (ns <= 1) return;
  double2 acc[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) acc[l] = make_double2(0, 0);
  for (int j = s0; j < s1; ++j) {
    int g = op.stab[j];
    bool neg = (chimask >> g) & 1ull;
    uint32_t sgm = op.sgm[g];
#pragma unroll
    for (int l = 0; l < 9; ++l) {
      // x[pi(l)] by selection over fixed indices: the node's values stay in registers (no dynamically indexed array)
      const int p = op.pi[g * 9 + l];
      double2 v = x[0];
#pragma unroll
      for (int q = 1; q < 9; ++q)
        if (q == p) v = x[q];
      if (((sgm >> l) & 1u) ^ (neg ? 1u : 0u)) v = make_double2(-v.x, -v.y);
      acc[l] = cadd(acc[l], v);
    }
  }
#pragma unroll
  for (int l = 0; l < 9; ++l) x[l] = cscale(acc[l], 1.0 / (double)ns);
}

// w = y - a u - b u' (projected) and the partials of w . w; w replaces y, or goes to wout when given (y kept)
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_lanczos_w(OpView op, BatchView bv, typename St2<ST>::T* __restrict__ y,
                                                        const typename St2<ST>::T* __restrict__ u,
                                                        const typename St2<ST>::T* __restrict__ up, double2* part, int npw,
                                                        typename St2<ST>::T* __restrict__ wout = nullptr) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = bv.lane_group[L];
  const bool act = grp >= 0 && bv.lane_wact[L];
  const unsigned long long chim = grp >= 0 ? bv.ginfo[grp].chimask : 0ull;
  const double2 a = bv.acur[L], b = bv.bprev[L], su = bv.su[L], sup = bv.sup[L];
  const double2 as = cmul(a, su), bs = cmul(b, sup);
  double2 dot = make_double2(0.0, 0.0);
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    double2 x[9];
    if (act) {
      for (int l = 0; l < 9; ++l) {
        size_t q = vix(it.tile, bv.nn, i, l) + lane;
        x[l] = csub(csub(ld_cs(y + q), cmul(as, ld(u + q))), cmul(bs, ld_cs(up + q)));
      }
      if (bv.project) project_node(op, i, chim, x);
      double2 dn = make_double2(0, 0);
      for (int l = 0; l < 9; ++l) dn = cadd(dn, cmul(x[l], x[l]));
      dot = cadd(dot, cscale(dn, op.sq[i] * op.sq[i]));
    } else {
      for (int l = 0; l < 9; ++l) x[l] = make_double2(0, 0);
    }
    typename St2<ST>::T* dst = wout ? wout : y;
    for (int l = 0; l < 9; ++l) stv(dst + vix(it.tile, bv.nn, i, l) + lane, x[l]);
  }
  block_reduce_store(dot, part, it.tile, bpt);
  if (bv.tick && last_block_of_tile(bv.tick, it.tile, bpt)) {
    const double2 ww = block_sum_rows(part + (size_t)it.tile * bpt * TL, bpt, TL);
    if (threadIdx.x < TL) reduce_b_lane(bv, ww, bv.kstep, 1.0e-12, it.tile, threadIdx.x, true);
  }
}

// in-place projection of a batch vector (asr_op_project_c)
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_project(OpView op, BatchView bv, typename St2<ST>::T* __restrict__ x, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = bv.lane_group[L];
  if (grp < 0) return;
  const unsigned long long chim = bv.ginfo[grp].chimask;
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    double2 v[9];
    for (int l = 0; l < 9; ++l) v[l] = ld(x + vix(it.tile, bv.nn, i, l) + lane);
    project_node(op, i, chim, v);
    for (int l = 0; l < 9; ++l) stv(x + vix(it.tile, bv.nn, i, l) + lane, v[l]);
  }
}

// ------------------------------------------------------------------------------------------------ per-lane scalars
// the per-tile reduction kernels: one block of RED_THREADS per tile (block_sum_rows), warp 0 finishes per lane
constexpr int RED_THREADS = WPB * TL;
__global__ void k_reduce_a(BatchView bv, const double2* part, int bpt, int k) {
  int tile = blockIdx.x;
  if (tile >= bv.ntile || !bv.tile_act[tile]) return;
  const double2 a = block_sum_rows(part + (size_t)tile * bpt * TL, bpt, TL);
  if (threadIdx.x < TL) reduce_a_lane<true>(bv, a, k, tile, threadIdx.x);
}

__global__ void k_reduce_b(BatchView bv, const double2* part, int bpt, int k, double btol) {
  int tile = blockIdx.x;
  if (tile >= bv.ntile) return;
  const bool live = bv.tile_act[tile] != 0;
  const double2 ww = live ? block_sum_rows(part + (size_t)tile * bpt * TL, bpt, TL) : make_double2(0, 0);
  if (threadIdx.x < TL) reduce_b_lane(bv, ww, k, btol, tile, threadIdx.x, live);
}

// final fraction of every lane: cf_species with the chosen tail (edc mode); lmap: batch lane -> output lane (-1: none)
__global__ void k_cf_final(BatchView bv, int nlane, const int* lmap, double2* g) {
  int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlane) return;
  int dst = lmap[L];
  if (bv.lane_group[L] < 0 || dst < 0) return;
  int m = bv.lane_m[L];
  double2 wd[NLMAX], we[NLMAX];
  int nf = 0;
  g[dst] = m > 0 ? cf_species_dev(bv.acoef + (size_t)L * NLMAX, bv.bcoef + (size_t)L * NLMAX, m, bv.lane_z[L], bv.tail, wd, we,
                                  &nf, nullptr)
                 : make_double2(0, 0);
  if (nf) atomicAdd(bv.nfall, nf);
}

// depths of the batch lanes into the run's array, and the energies of the batch lanes from the run's array
__global__ void k_scatter_m(int nlane, const int* lmap, const int* m, int* m_all) {
  int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L < nlane && lmap[L] >= 0) m_all[lmap[L]] = m[L];
}
__global__ void k_gather_z(int nlane, const int* lmap, const double2* z_all, double2* z) {
  int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L < nlane) z[L] = lmap[L] >= 0 ? z_all[lmap[L]] : make_double2(0.0, 0.0);
}

// projections of u_k on the target states (edc_green_proj, src/asr_edc.f90:196-202): one warp per (tile, target),
// cpr(k, l, t) = sum_ks tw(l, ks, t) psi(node ks of t, l) with psi = chi(g) sg(l, g) u(r, pi(l, g)) in amplitude
// coordinates (augcls_amp_c, src/asr_augcls.f90:251-261: the normalised v(r) over sqrt(orbit size)), times the lane
// scale of the stored vector
template <typename ST>
__global__ void k_proj_gather(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ u, ProjView P, int k) {
  const int lane = threadIdx.x % TL;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) / TL;
  const int tile = (int)(warp / P.nt), t = (int)(warp % P.nt);
  if (tile >= bv.ntile) return;
  const int L = tile * TL + lane;
  const int grp = bv.lane_group[L];
  double2 acc[9];
  for (int l = 0; l < 9; ++l) acc[l] = make_double2(0.0, 0.0);
  if (grp >= 0) {
    const double2 su = bv.su[L];
    const unsigned long long chim = bv.ginfo[grp].chimask;
    const double* tw = P.tw + ((size_t)grp * P.nt + t) * 9 * P.nsm;
    for (int ks = 0; ks < P.nsm; ++ks) {
      const int r = P.tnode[ks + P.nsm * t];
      if (r < 0) continue;
      const int g = P.tgop[ks + P.nsm * t];
      const double chi = ((chim >> g) & 1ull) ? -1.0 : 1.0;
      const unsigned sgm = op.sgm[g];
      for (int l = 0; l < 9; ++l) {
        const int pl = op.pi[l + 9 * g];
        const double wgt = tw[l + 9 * ks] * chi * (((sgm >> l) & 1u) ? -1.0 : 1.0);
        const double2 x = ld(u + vix(tile, bv.nn, r, pl) + lane);
        acc[l] = cadd(acc[l], cscale(x, wgt));
      }
    }
    for (int l = 0; l < 9; ++l) acc[l] = cmul(acc[l], su);
  }
  double2* dst = P.cpr + (((size_t)tile * P.kcap + (k - 1)) * 9 * P.nt + (size_t)t * 9) * TL + lane;
  for (int l = 0; l < 9; ++l) dst[(size_t)l * TL] = acc[l];
}

// gp(l, t) = sum_k cpr(k, l, t) pv_k with pv of cf_species at depth m, and gp4 the same at max(1, m - 4)
// (src/asr_edc.f90:221-231); one thread per lane
__global__ void k_proj_final(BatchView bv, int nlane, const int* lmap, ProjView P) {
  int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlane) return;
  int dst = lmap[L];
  if (bv.lane_group[L] < 0 || dst < 0) return;
  const int tile = L / TL, lane = L % TL, m = bv.lane_m[L];
  double2 pv[NLMAX], wd[NLMAX], we[NLMAX];
  int nf = 0;
  for (int pass = 0; pass < 2; ++pass) {
    double2* out = (pass == 0 ? P.gp : P.gp4) + (size_t)dst * P.nt * 9;
    const int mm = pass == 0 ? m : (m - 4 > 1 ? m - 4 : 1);
    if (m < 1) {
      for (int q = 0; q < 9 * P.nt; ++q) out[q] = make_double2(0.0, 0.0);
      continue;
    }
    cf_species_pv_dev(bv.acoef + (size_t)L * NLMAX, bv.bcoef + (size_t)L * NLMAX, mm, bv.lane_z[L], bv.tail, pv, wd, we,
                      pass == 0 ? &nf : nullptr);
    for (int q = 0; q < 9 * P.nt; ++q) {
      double2 acc = make_double2(0.0, 0.0);
      for (int kk = 0; kk < mm; ++kk)
        acc = cadd(acc, cmul(P.cpr[(((size_t)tile * P.kcap + kk) * 9 * P.nt + q) * TL + lane], pv[kk]));
      out[q] = acc;
    }
  }
  if (nf) atomicAdd(bv.nfall, nf);
}

// start vectors: U = e_(node 0, l0) with scale 1, UP = 0
template <typename ST>
__global__ void k_init(BatchView bv, typename St2<ST>::T* u, typename St2<ST>::T* up) {
  size_t n = (size_t)bv.ntile * bv.nn * 9 * TL;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int lane = (int)(q % TL);
    size_t rest = q / TL;
    int l = (int)(rest % 9);
    size_t nt = rest / 9;
    int node = (int)(nt % bv.nn);
    int tile = (int)(nt / bv.nn);
    int L = tile * TL + lane;
    int grp = bv.lane_group[L];
    double v = (grp >= 0 && node == 0 && l == bv.ginfo[grp].l0 - 1) ? 1.0 : 0.0;
    stv(u + q, make_double2(v, 0.0));
    stv(up + q, make_double2(0.0, 0.0));
  }
}

size_t smul_smem(const asr_op* op, size_t st_size) {
  size_t b = (size_t)op->ntype * (op->nslot + 1) * 9 * RW * st_size;
  b = (b + 15) & ~(size_t)15;
  b += (size_t)op->nop * sizeof(unsigned long long);
  return b;
}

// the staged (bulk-copy) S application when ASR_SMUL_BULK=1.  Measured on the fcc ternary workload it is slower than
// the direct gathers (FP64 5.3 / 7.1 / 7.4 ms per 16-tile launch with 2 / 3 / 4 stages against 4.55 ms; FP32 1.72 ms
// against 1.35 ms): the per-node rows are small copies, and the stage buffers cost the occupancy that hides the gathers
bool smul_bulk_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("ASR_SMUL_BULK");
    on = (e && atoi(e) == 1) ? 1 : 0;
  }
  return on == 1;
}

template <typename ST, bool FUSE_D, bool FINAL, int EPI = 0>
void launch_smul(asr_op* op, const BatchView& bv, const ST* blk, const typename St2<ST>::T* in, typename St2<ST>::T* out,
                 double2* part, int npw, int grid, cudaStream_t s) {
  OpView ov = op->view();
  const int pix = std::is_same<ST, double>::value ? 0 : 1;
  if (EPI) {   // the adjoint's fused steps: also t2 (bv.t2out); EPI 2, the reverse epilogue (bv.adj)
    if (op->tuned_link[pix] == 1)
      k_smul<ST, FUSE_D, FINAL, true, EPI><<<grid, WPB * TL, smul_smem(op, sizeof(ST)), s>>>(ov, bv, blk, in, out, part, npw);
    else
      k_smul<ST, FUSE_D, FINAL, false, EPI><<<grid, WPB * TL, smul_smem(op, sizeof(ST)), s>>>(ov, bv, blk, in, out, part, npw);
    return;
  }
  if (smul_bulk_enabled())
    k_smul_bulk<ST, FUSE_D, FINAL><<<grid, WPB * TL, smul_bulk_smem<ST>(op), s>>>(ov, bv, blk, in, out, part, npw, op->ctx->d_err);
  else if (op->tuned_link[pix] == 1)
    k_smul<ST, FUSE_D, FINAL, true><<<grid, WPB * TL, smul_smem(op, sizeof(ST)), s>>>(ov, bv, blk, in, out, part, npw);
  else
    k_smul<ST, FUSE_D, FINAL, false><<<grid, WPB * TL, smul_smem(op, sizeof(ST)), s>>>(ov, bv, blk, in, out, part, npw);
}

// a bounded wait of the staged kernels that ran out (the device error word), as a status
int check_wait_error(asr_ctx* ctx) {
  int h = 0;
  ASR_CUDA(cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  ASR_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h == DERR_WAIT) {
    cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream);
    set_error("chains: a bulk copy of the staged operator did not complete in time");
    return ASR_ESTATE;
  }
  return ASR_OK;
}

// One chain step of the general operator on the batch; writes y into Y and the a-partials.
template <typename ST>
int step_apply(asr_ctx* ctx, asr_op* op, const BatchView& bv, bool fused, bool any_o, bool all_dunif,
               typename St2<ST>::T* U, typename St2<ST>::T* Y, typename St2<ST>::T* T1, typename St2<ST>::T* T2,
               typename St2<ST>::T* H1, typename St2<ST>::T* R1, double2* part, int npw, int grid) {
  cudaStream_t s = ctx->stream;
  OpView ov = op->view();
  const ST* blk = std::is_same<ST, double>::value ? (const ST*)op->d_blocks : (const ST*)op->d_blocks_f;
  size_t sm = smul_smem(op, sizeof(ST));
  dim3 B(WPB * TL);
  if (fused) {
    launch_smul<ST, true, true>(op, bv, blk, U, Y, part, npw, grid, s);
    return ASR_OK;
  }
  // t1 = D x0, t2 = S t1
  if (all_dunif) {
    launch_smul<ST, true, false>(op, bv, blk, U, T2, part, npw, grid, s);
  } else {
    k_rand<ST><<<grid, B, 0, s>>>(ov, bv, PD, U, T1, npw);
    launch_smul<ST, false, false>(op, bv, blk, T1, T2, part, npw, grid, s);
  }
  if (!any_o) {   // y = s (D t2 + (c + e + X) U)
    k_combine<ST><<<grid, B, 0, s>>>(ov, bv, T2, U, PCEB, true, U, false, nullptr, 1.0, true, Y, part, npw);
    return ASR_OK;
  }
  // h1 = D t2 + C U;  r1 = O h1;  h2 = D S D r1 + C r1;  y = s (h1 - h2 + (e + X) U)
  k_combine<ST><<<grid, B, 0, s>>>(ov, bv, T2, U, PC, false, U, false, nullptr, 1.0, false, H1, part, npw);
  k_rand<ST><<<grid, B, 0, s>>>(ov, bv, PO, H1, R1, npw);
  k_rand<ST><<<grid, B, 0, s>>>(ov, bv, PD, R1, T1, npw);
  launch_smul<ST, false, false>(op, bv, blk, T1, T2, part, npw, grid, s);
  k_combine<ST><<<grid, B, 0, s>>>(ov, bv, T2, R1, PC, false, U, true, H1, -1.0, true, Y, part, npw);
  return ASR_OK;
}

// The vector memory of a batched run as one slab: the context's held slab (asr_ctx_hold_workspace; grown when too small
// and kept after the call), else `own`, allocated here and freed with the caller's scope.  Calls on one context run in
// its stream order and return after their last kernel, so a held slab is never in use by two calls.
int vector_slab(asr_ctx* ctx, size_t bytes, Dev<unsigned char>& own, void** base) {
  if (ctx->ws_hold) {
    if (ctx->ws_bytes < bytes) {
      ctx->ws_release();
      if (cudaMalloc(&ctx->ws, bytes) != cudaSuccess) {
        ctx->ws = nullptr;
        set_error("chains: device allocation of %zu bytes failed", bytes);
        return ASR_ENOMEM;
      }
      ctx->ws_bytes = bytes;
    }
    *base = ctx->ws;
    return ASR_OK;
  }
  ASR_TRY(own.alloc(bytes));
  *base = own.p;
  return ASR_OK;
}

template <typename ST>
int run_lanes_t(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                const GroupLayout& GL, const std::vector<int>& lane_group, const double2* d_lane_z, int nlane,
                const RunOptions& opt, double2* d_g_out, std::vector<double2>* a_out, std::vector<double2>* b_out,
                std::vector<int>* m_out, int64_t* nfall_out, int64_t* nsteps_out, const ProjSpec* proj, double* dev_ms) {
  typedef typename St2<ST>::T T2;
  cudaStream_t s = ctx->stream;
  const int nn = op->nn;
  // tiles: the lanes of one group in chunks of 32 (a tile never holds two groups)
  std::vector<std::vector<int>> tiles;
  {
    std::vector<std::vector<int>> per_group(ginfo.size());
    for (int L = 0; L < nlane; ++L) per_group[lane_group[L]].push_back(L);
    for (auto& lst : per_group)
      for (size_t q = 0; q < lst.size(); q += TL)
        tiles.emplace_back(lst.begin() + q, lst.begin() + std::min(lst.size(), q + (size_t)TL));
  }
  const int ntile_all = (int)tiles.size();
  int nlevmax = 0;
  bool any_o = false, all_dunif = true, fused = true;
  for (auto& g : ginfo) {
    nlevmax = std::max(nlevmax, g.nlev);
    if (!(g.flags & GF_O_ZERO)) any_o = true;
    if (!(g.flags & GF_D_UNIFORM)) all_dunif = false;
  }
  fused = all_dunif && !any_o;
  if (nlevmax > NLMAX) { set_error("chains: depth %d above the device maximum %d", nlevmax, NLMAX); return ASR_EINVAL; }
  if (op->nop > MAXOP) { set_error("chains: at most %d group operations", MAXOP); return ASR_EINVAL; }
  // batch size: tiles in flight, bounded by memory (3 vectors + temporaries per tile)
  const size_t vec_bytes = (size_t)nn * 9 * TL * sizeof(T2);
  const int nvec = 3 + (fused ? 0 : (any_o ? 4 : 2));
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  freeb += ctx->ws_bytes;   // a held slab is this call's to reuse
  // 32-lane tiles per batch: larger batches amortise the per-level reductions and launch gaps; the caller's shape, else
  // the operator's autotuned one, else the measured defaults of the fcc ternary workload (FP64 16 tiles, FP32 8, 4 nodes
  // per warp)
  const int prec_ix = std::is_same<ST, double>::value ? 0 : 1;
  int tpb = opt.tiles_per_batch > 0 ? opt.tiles_per_batch
          : op->tuned_tpb[prec_ix] > 0 ? op->tuned_tpb[prec_ix] : (std::is_same<ST, double>::value ? 16 : 8);
  if (const char* e = getenv("ASR_TILES_PER_BATCH")) tpb = std::max(1, atoi(e));
  // projections: per tile nlevmax x 9 nt x 32 complex values
  const size_t proj_tile_bytes = proj ? (size_t)nlevmax * 9 * proj->nt * TL * sizeof(double2) : 0;
  while (tpb > 1 && (size_t)tpb * (nvec * vec_bytes + proj_tile_bytes) > freeb / 2) tpb /= 2;
  tpb = std::min(tpb, ntile_all);
  int npw = opt.nodes_per_warp > 0 ? opt.nodes_per_warp : op->tuned_npw[prec_ix] > 0 ? op->tuned_npw[prec_ix] : 4;
  if (const char* e = getenv("ASR_NODES_PER_WARP")) npw = std::max(1, atoi(e));
  const int npb = WPB * npw;
  const int bpt = (nn + npb - 1) / npb;
  // device state
  Dev<double> d_gblob;
  Dev<GroupInfo> d_ginfo;
  ASR_TRY(d_gblob.alloc(gblob.size()));
  ASR_TRY(d_ginfo.alloc(ginfo.size()));
  ASR_CUDA(cudaMemcpyAsync(d_gblob.p, gblob.data(), gblob.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_ginfo.p, ginfo.data(), ginfo.size() * sizeof(GroupInfo), cudaMemcpyHostToDevice, s));
  const int nlp = tpb * TL;
  Dev<int> d_lgroup, d_act, d_wact, d_m, d_tact, d_nfall, d_tgroup, d_tick;
  Dev<double2> d_a, d_b, d_gprev, d_acur, d_bprev, d_su, d_sup, d_part, d_z;
  ASR_TRY(d_lgroup.alloc(nlp)); ASR_TRY(d_act.alloc(nlp)); ASR_TRY(d_wact.alloc(nlp)); ASR_TRY(d_m.alloc(nlp));
  ASR_TRY(d_tact.alloc(tpb)); ASR_TRY(d_nfall.alloc(1)); ASR_TRY(d_tgroup.alloc(tpb)); ASR_TRY(d_tick.alloc(tpb));
  ASR_TRY(d_a.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_b.alloc((size_t)nlp * NLMAX));
  ASR_TRY(d_gprev.alloc(nlp)); ASR_TRY(d_acur.alloc(nlp)); ASR_TRY(d_bprev.alloc(nlp)); ASR_TRY(d_su.alloc(nlp));
  ASR_TRY(d_sup.alloc(nlp)); ASR_TRY(d_part.alloc((size_t)tpb * bpt * TL)); ASR_TRY(d_z.alloc(nlp));
  const size_t vlen = (size_t)tpb * nn * 9 * TL;
  Dev<unsigned char> own;
  T2* vbase = nullptr;
  ASR_TRY(vector_slab(ctx, (size_t)nvec * vlen * sizeof(T2), own, (void**)&vbase));
  struct VecRef { T2* p; };
  VecRef V[7];
  for (int q = 0; q < nvec; ++q) V[q].p = vbase + (size_t)q * vlen;
  Dev<double2> d_cpr;
  ProjView PV{0, 1, nlevmax, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  if (proj) {
    ASR_TRY(d_cpr.alloc((size_t)tpb * nlevmax * 9 * proj->nt * TL));
    PV = ProjView{proj->nt, proj->nsm, nlevmax, proj->tnode, proj->tgop, proj->tw, d_cpr.p, proj->gp, proj->gp4};
  }
  ASR_CUDA(cudaMemsetAsync(d_nfall.p, 0, sizeof(int), s));
  if (a_out) { a_out->assign((size_t)nlane * NLMAX, make_double2(0, 0)); b_out->assign((size_t)nlane * NLMAX, make_double2(0, 0)); }
  if (m_out) m_out->assign(nlane, 0);
  std::vector<int> hgroup(nlp), lmap(nlp), hm_all(nlane, 0);
  std::vector<double2> ha, hb;
  Dev<int> d_lmap, d_m_all;
  ASR_TRY(d_lmap.alloc(nlp));
  ASR_TRY(d_m_all.alloc(nlane));
  ASR_CUDA(cudaMemsetAsync(d_m_all.p, 0, nlane * sizeof(int), s));
  // deepest tiles first, so that every batch runs to one depth
  std::vector<int> tdepth(ntile_all, 0), order(ntile_all);
  for (int t = 0; t < ntile_all; ++t) tdepth[t] = ginfo[lane_group[tiles[t][0]]].nlev;
  for (int t = 0; t < ntile_all; ++t) order[t] = t;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tdepth[x] > tdepth[y]; });
  std::vector<double2> one(nlp, make_double2(1.0, 0.0));
  cudaEvent_t tev[2] = {nullptr, nullptr};   // device time of the batches (after the allocations), for the autotuner
  if (dev_ms) {
    ASR_CUDA(cudaEventCreate(&tev[0]));
    ASR_CUDA(cudaEventCreate(&tev[1]));
    ASR_CUDA(cudaEventRecord(tev[0], s));
  }
  for (int t0 = 0; t0 < ntile_all; t0 += tpb) {
    NvtxRange batch_range("chain batch");
    const int nt = std::min(tpb, ntile_all - t0);
    int kmax = 0;
    std::vector<int> tact(tpb, 0), ones(nlp, 0), tgroup(tpb, -1);
    for (int q = 0; q < nlp; ++q) {
      int bt = q / TL;
      int L = -1;
      if (bt < nt) {
        const std::vector<int>& tl = tiles[order[t0 + bt]];
        if (q % TL < (int)tl.size()) L = tl[q % TL];
      }
      lmap[q] = L;
      hgroup[q] = L >= 0 ? lane_group[L] : -1;
      if (hgroup[q] >= 0) { kmax = std::max(kmax, ginfo[hgroup[q]].nlev); tact[bt] = 1; ones[q] = 1; tgroup[bt] = hgroup[q]; }
    }
    ASR_CUDA(cudaMemcpyAsync(d_tgroup.p, tgroup.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_lgroup.p, hgroup.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_lmap.p, lmap.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_act.p, ones.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tact.p, tact.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemsetAsync(d_wact.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_tick.p, 0, tpb * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_m.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_a.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_b.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_gprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_bprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_sup.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemcpyAsync(d_su.p, one.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    k_gather_z<<<(nlp + 127) / 128, 128, 0, s>>>(nlp, d_lmap.p, d_lane_z, d_z.p);
    BatchView bv{nt, nn, op->nsmax, 0, opt.mode, opt.project, opt.tail, NLMAX, opt.depth_tol, d_gblob.p, GL, d_ginfo.p,
                 d_lgroup.p, d_tgroup.p, d_z.p, d_act.p, d_wact.p, d_m.p, d_a.p, d_b.p, d_gprev.p, d_acur.p, d_bprev.p, d_su.p,
                 d_sup.p, d_tact.p, d_nfall.p};
    k_init<ST><<<std::min<size_t>(65535, ((size_t)nt * nn * 9 * TL + 255) / 256), 256, 0, s>>>(bv, V[1].p, V[0].p);
    ctx->launches += 2;
    const int gridb = nt * bpt;
    for (int k = 1; k <= kmax; ++k) {
      bv.kstep = k;
      T2* U = V[k % 3].p;
      T2* UP = V[(k + 2) % 3].p;
      T2* Y = V[(k + 1) % 3].p;
      if (proj) {   // projections of u_k before the operator step (src/asr_edc.f90:196-202)
        const long nwarp = (long)nt * proj->nt;
        k_proj_gather<ST><<<(unsigned)((nwarp * TL + 255) / 256), 256, 0, s>>>(op->view(), bv, U, PV, k);
        ctx->launches += 1;
      }
      // the fused step reduces a_k in its epilogue (the tile's last block), except at the levels of the depth test, whose
      // fraction evaluation runs in the separate reduction kernel; k_lanczos_w always reduces b_k in its epilogue
      const bool depth_due = opt.depth_tol > 0.0 && opt.mode == ASR_MODE_EDC && k >= 8 && k % 4 == 0;
      const bool a_in_step = fused && !depth_due;
      BatchView bvs = bv;
      bvs.tick = a_in_step ? d_tick.p : nullptr;
      // timed regions (asr_ctx_profile): event pairs stay pending until the statistics are read (no synchronisation)
      int ps = ctx->prof_start(s);
      ASR_TRY(step_apply<ST>(ctx, op, bvs, fused, any_o, all_dunif, U, Y, nvec > 3 ? V[3].p : nullptr, nvec > 3 ? V[4].p : nullptr,
                             nvec > 5 ? V[5].p : nullptr, nvec > 5 ? V[6].p : nullptr, d_part.p, npw, gridb));
      {   // algorithmic traffic of one operator pass: read U and write Y per (node, lane), plus the node tables per tile
        const double tab = (double)op->nslot * 5 + (double)op->nsmax * 5 + 8 + 8 + 4;
        ctx->prof_stop(s, ps, ASR_KERNEL_STEP, (double)nt * nn * (2.0 * 9 * TL * sizeof(T2) + tab),
                       (double)nt * nn * TL * (op->nslot + 1) * 81.0 * 4.0);
      }
      if (!a_in_step) k_reduce_a<<<nt, RED_THREADS, 0, s>>>(bv, d_part.p, bpt, k);
      BatchView bvw = bv;
      bvw.tick = d_tick.p;
      ps = ctx->prof_start(s);
      k_lanczos_w<ST><<<gridb, WPB * TL, 0, s>>>(op->view(), bvw, Y, U, UP, d_part.p, npw);
      // read y, u, u', write w per (node, lane); about 30 flops per complex element (scaled updates, projection, dot)
      ctx->prof_stop(s, ps, ASR_KERNEL_LANCZOS, (double)nt * nn * 4.0 * 9 * TL * sizeof(T2), (double)nt * nn * TL * 9 * 30.0);
      ctx->launches += (a_in_step ? 1 : 2) + (fused ? 1 : (any_o ? 7 : (all_dunif ? 2 : 3)));
    }
    ASR_CUDA(cudaGetLastError());
    if (opt.mode == ASR_MODE_EDC && d_g_out) {
      k_cf_final<<<(nlp + 63) / 64, 64, 0, s>>>(bv, nlp, d_lmap.p, d_g_out);
      ctx->launches += 1;
    }
    if (proj && opt.mode == ASR_MODE_EDC) {
      k_proj_final<<<(nlp + 63) / 64, 64, 0, s>>>(bv, nlp, d_lmap.p, PV);
      ctx->launches += 1;
    }
    k_scatter_m<<<(nlp + 127) / 128, 128, 0, s>>>(nlp, d_lmap.p, d_m.p, d_m_all.p);
    ctx->launches += 2;
    if (a_out) {   // coefficients back to the host (tests): synchronise this batch
      ha.resize((size_t)nlp * NLMAX); hb.resize((size_t)nlp * NLMAX);
      ASR_CUDA(cudaMemcpyAsync(ha.data(), d_a.p, (size_t)nlp * NLMAX * sizeof(double2), cudaMemcpyDeviceToHost, s));
      ASR_CUDA(cudaMemcpyAsync(hb.data(), d_b.p, (size_t)nlp * NLMAX * sizeof(double2), cudaMemcpyDeviceToHost, s));
      ASR_CUDA(cudaStreamSynchronize(s));
      ASR_CUDA(cudaGetLastError());
        for (int q = 0; q < nlp; ++q) {
          int L = lmap[q];
          if (L < 0) continue;
          std::memcpy(&(*a_out)[(size_t)L * NLMAX], &ha[(size_t)q * NLMAX], NLMAX * sizeof(double2));
          std::memcpy(&(*b_out)[(size_t)L * NLMAX], &hb[(size_t)q * NLMAX], NLMAX * sizeof(double2));
        }
    }
  }
  if (dev_ms) {
    ASR_CUDA(cudaEventRecord(tev[1], s));
    ASR_CUDA(cudaEventSynchronize(tev[1]));
    float ms = 0.f;
    ASR_CUDA(cudaEventElapsedTime(&ms, tev[0], tev[1]));
    *dev_ms = ms;
    cudaEventDestroy(tev[0]);
    cudaEventDestroy(tev[1]);
  }
  ASR_CUDA(cudaMemcpyAsync(hm_all.data(), d_m_all.p, nlane * sizeof(int), cudaMemcpyDeviceToHost, s));
  int64_t nsteps = 0;
  int nf = 0;
  ASR_CUDA(cudaMemcpyAsync(&nf, d_nfall.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  ASR_TRY(check_wait_error(ctx));
  for (int L = 0; L < nlane; ++L) nsteps += hm_all[L];
  if (m_out) *m_out = hm_all;
  if (nfall_out) *nfall_out = nf;
  if (nsteps_out) *nsteps_out = nsteps;
  return ASR_OK;
}

// ================================================================================================ adjoint
// Reverse mode through the chain (the derivative of the computed G, not of the exact resolvent), for the edc route
// with o = 0 and a fixed depth.  Forward: u_1 = e, y_k = A u_k, a_k = u_k . y_k, w_k = y_k - a_k u_k - b_{k-1} u_{k-1},
// w'_k = P w_k, b_k = sqrt(w'_k . w'_k), u_{k+1} = w'_k / b_k; G = cf(a, b).  With the bilinear form of the normalised
// coordinates (amplitude coordinates weighted by the orbit size) A and P are symmetric on the symmetric subspace, and
// every quantity is holomorphic in the parameters, so the adjoint recursion for the seeds abar_k, bbar_k is
//   bbar_k -= (ubar_{k+1} . u_{k+1}) / b_k;  wbar = P (ubar_{k+1} / b_k + bbar_k u_{k+1})
//   abar_k -= wbar . u_k;  bbar_{k-1} -= wbar . u_{k-1};  ybar = wbar + abar_k u_k
//   ubar_k += A ybar + abar_k y_k - a_k wbar;  ubar_{k-1} -= b_{k-1} wbar;  theta_bar += ybar . (dA/dtheta) u_k.
// For A = R_d S R_d + R_P (amplitude coordinates), ybar . dA u = ybar . dR_P u + ybar . dR_d (S R_d u) + (S R_d ybar) . dR_d u,
// and dR_p / dpar(l, s) is the random operator with the weights mt(own, k', s, class) (local_weights,
// src/asr_augcls.f90:362-377).  The Lanczos vectors are recomputed per segment from checkpoints every `stride` levels.

constexpr int MAXSP = 8;        // species of the gradient kernel's register accumulators (at most)
constexpr int GPW = 9;          // warps per gradient block: one per orbital

// per-lane weighted dot: part = sum_i norb_i a_i . b_i (raw, unscaled vectors)
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_dot(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ a,
                                                  const typename St2<ST>::T* __restrict__ b, double2* part, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  double2 dot = make_double2(0, 0);
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    double2 dn = make_double2(0, 0);
    for (int l = 0; l < 9; ++l) {
      size_t q = vix(it.tile, bv.nn, i, l) + lane;
      dn = cadd(dn, cmul(ld(a + q), ld(b + q)));
    }
    dot = cadd(dot, cscale(dn, op.sq[i] * op.sq[i]));
  }
  block_reduce_store(dot, part, it.tile, bpt);
}

// wbar = P (c1 ubar_next + c2 X_next); partial dots wbar . X_k and wbar . X_{k-1}
template <typename ST>
__global__ void __launch_bounds__(WPB * TL, 2) k_adj_w(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ ubn,
                                                    const typename St2<ST>::T* __restrict__ xn, const typename St2<ST>::T* __restrict__ xk,
                                                    const typename St2<ST>::T* __restrict__ xkm, const double2* c1, const double2* c2,
                                                    typename St2<ST>::T* __restrict__ wb, double2* part1, double2* part2, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = bv.lane_group[L];
  const unsigned long long chim = grp >= 0 ? bv.ginfo[grp].chimask : 0ull;
  const double2 a1 = c1[L], a2 = c2[L];
  double2 d1 = make_double2(0, 0), d2 = make_double2(0, 0);
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    double2 x[9];
    for (int l = 0; l < 9; ++l) {
      size_t q = vix(it.tile, bv.nn, i, l) + lane;
      x[l] = cadd(cmul(a1, ld(ubn + q)), cmul(a2, ld(xn + q)));
    }
    if (bv.project) project_node(op, i, chim, x);
    double2 e1 = make_double2(0, 0), e2 = make_double2(0, 0);
    for (int l = 0; l < 9; ++l) {
      size_t q = vix(it.tile, bv.nn, i, l) + lane;
      stv(wb + q, x[l]);
      e1 = cadd(e1, cmul(x[l], ld(xk + q)));
      e2 = cadd(e2, cmul(x[l], ld(xkm + q)));
    }
    double nb = op.sq[i] * op.sq[i];
    d1 = cadd(d1, cscale(e1, nb));
    d2 = cadd(d2, cscale(e2, nb));
  }
  block_reduce_store(d1, part1, it.tile, bpt);
  __syncthreads();
  block_reduce_store(d2, part2, it.tile, bpt);
}

// ybar = wbar + c3 X_k;  ubar_{k-1} -= c4 wbar
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_adj_y(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ wb,
                                                    const typename St2<ST>::T* __restrict__ xk, const double2* c3, const double2* c4,
                                                    typename St2<ST>::T* __restrict__ yb, typename St2<ST>::T* __restrict__ ubp, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const double2 a3 = c3[L], a4 = c4[L];
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    for (int l = 0; l < 9; ++l) {
      size_t q = vix(it.tile, bv.nn, i, l) + lane;
      double2 wv = ld(wb + q);
      stv(yb + q, cadd(wv, cmul(a3, ld(xk + q))));
      if (ubp) stv(ubp + q, csub(ld(ubp + q), cmul(a4, wv)));
    }
  }
}

// ubar_k += AY + c5 Y_k - c6 wbar
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_adj_u(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ ay,
                                                    const typename St2<ST>::T* __restrict__ yk, const typename St2<ST>::T* __restrict__ wb,
                                                    const double2* c5, const double2* c6, typename St2<ST>::T* __restrict__ ubk, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const double2 a5 = c5[L], a6 = c6[L];
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    for (int l = 0; l < 9; ++l) {
      size_t q = vix(it.tile, bv.nn, i, l) + lane;
      double2 v = cadd(ld(ubk + q), ld(ay + q));
      v = cadd(v, cmul(a5, ld(yk + q)));
      v = csub(v, cmul(a6, ld(wb + q)));
      stv(ubk + q, v);
    }
  }
}

// gradient partials of one reverse step: thread (orbital l = warp, lane); per block and kind the sums over its nodes and
// the 32 lanes: gpart[((tile * gbpt + blk) * NGK + kind) * 9 * nsp + l * nsp + species], kinds 0 c, 1 d, 2 pa, 3 o, 4 e
// (e and pb enter the same way).  With G_p(x, v) = x . (dR_p / dpar) v (x at the node, v through the flip links with the
// class weights mt, or the node itself on a frozen site) and A = h - h O h + E + X(z), h = C + D S D:
//   c: G(yb, u) - G(yb, O h u) - G(O h yb, u)
//   d: Gh(yb, u) - Gh(yb, O h u) - Gh(O h yb, u),  Gh(x, v) = G_d(x, S D v) + G_d(S D x, v)
//   o: -G(h yb, h u);  e: G(yb, u);  pa: z G(yb, u)
// GEN = false (O = 0): the last two terms of c and d and the o kind vanish, and the operator's intermediates are not read.
constexpr int NGK = 5;
struct AdjVecs {   // per level: node side (yb: ybar; tb = S D ybar; hb = h ybar; rb = O h ybar; qb = S D O h ybar) and link
                   // side (unscaled X_k; tk = S D X_k; hk = h X_k; rk = O h X_k; qk = S D O h X_k)
  const void *yb, *tb, *hb, *rb, *qb;
  const void *xk, *tk, *hk, *rk, *qk;
};
// a[sp] += v with sp known only at run time: an unrolled select over the NS accumulators keeps them in registers (an
// indexed array would live in local memory); the accumulator sees the same additions in the same order
template <int NS>
__device__ __forceinline__ void add_sp(double2 (&a)[NS], int sp, double2 v) {
#pragma unroll
  for (int q = 0; q < NS; ++q)
    if (q == sp) a[q] = cadd(a[q], v);
}

// NS: a compile-time bound on the operator's species count (nsp <= NS), which sizes the register accumulators
template <typename ST, bool GEN, bool WY = false, int NS = MAXSP>
__global__ void __launch_bounds__(GPW * TL) k_adj_grad(OpView op, BatchView bv, const double* mt, const int* spc, int ldspc,
                                                       AdjVecs V, const double2* sk, int nodes_per_block, double2* gpart,
                                                       const double2* cy = nullptr) {
  typedef typename St2<ST>::T T2;
  const T2 *yb = (const T2*)V.yb, *tb = (const T2*)V.tb, *hb = (const T2*)V.hb, *rb = (const T2*)V.rb, *qb = (const T2*)V.qb;
  const T2 *xk = (const T2*)V.xk, *tk = (const T2*)V.tk, *hk = (const T2*)V.hk, *rk = (const T2*)V.rk, *qk = (const T2*)V.qk;
  const int gbpt = (bv.nn + nodes_per_block - 1) / nodes_per_block;
  const int tile = blockIdx.x / gbpt, blk = blockIdx.x % gbpt;
  if (tile >= bv.ntile || !bv.tile_act[tile]) return;
  const int l = threadIdx.x / TL, lane = threadIdx.x % TL;
  const int L = tile * TL + lane;
  const int grp = bv.tile_group[tile];
  const int nsp = op.nsp, nsm = op.nsmax;
  double2 gc[NS], gd[NS], ge[NS], go[NS];   // pa = z e-kind
#pragma unroll
  for (int q = 0; q < NS; ++q) { gc[q] = make_double2(0, 0); gd[q] = gc[q]; ge[q] = gc[q]; go[q] = gc[q]; }
  const bool live = bv.lane_group[L] >= 0 && grp >= 0;
  double2 z = make_double2(0, 0);
  if (live) {
    const GroupInfo gi = bv.ginfo[grp];
    const double2 s = sk[L];
    const double2 c3 = WY ? cy[L] : make_double2(0, 0);
    z = bv.lane_z[L];
    const int i0 = blk * nodes_per_block, i1 = min(bv.nn, i0 + nodes_per_block);
    for (int i = i0; i < i1; ++i) {
      size_t q = vix(tile, bv.nn, i, l) + lane;
      double2 y = ld(yb + q), ty = ld(tb + q);
      if (WY) {   // the fused reverse step passes wbar and S D wbar: ybar = wbar + c3 X_k, S D ybar = S D wbar + c3 S D X_k
        y = cadd(y, cmul(c3, ld(xk + q)));
        ty = cadd(ty, cmul(c3, ld(tk + q)));
      }
      double2 hy = make_double2(0, 0), ry = hy, qy = hy;
      if (GEN) { hy = ld(hb + q); ry = ld(rb + q); qy = ld(qb + q); }
      const double nb = op.sq[i] * op.sq[i];
      const int fs = frozen_of(op, gi, i);
      const int kap = op.ncl[i], own = op.lst[i], nk = op.nsc[kap];
      const int nlink = fs > 0 ? 1 : nk;
      for (int kp = 0; kp < nlink; ++kp) {
        size_t qr = q;
        double sgn = 1.0;
        if (fs == 0 && kp != own) {
          int r = op.flipr[kp + nsm * i];
          if (r < 0) continue;
          int g = op.flipg[kp + nsm * i];
          bool neg = (gi.chimask >> g) & 1ull;
          sgn = ((((uint32_t)op.sgm[g] >> l) & 1u) ^ (neg ? 1u : 0u)) ? -1.0 : 1.0;
          qr = vix(tile, bv.nn, r, op.pi[g * 9 + l]) + lane;
        }
        const double2 x = cscale(cmul(s, ld(xk + qr)), sgn), t = cscale(cmul(s, ld(tk + qr)), sgn);
        double2 qe = cmul(y, x);                                          // G(yb, u)
        double2 qc = qe, qd = cadd(cmul(y, t), cmul(ty, x)), qo = make_double2(0, 0);
        if (GEN) {
          const double2 hx = cscale(cmul(s, ld(hk + qr)), sgn), rx = cscale(cmul(s, ld(rk + qr)), sgn);
          const double2 qx = cscale(cmul(s, ld(qk + qr)), sgn);
          qc = csub(csub(qe, cmul(y, rx)), cmul(ry, x));
          qd = csub(csub(qd, cadd(cmul(y, qx), cmul(ty, rx))), cadd(cmul(ry, t), cmul(qy, x)));
          qo = csub(make_double2(0, 0), cmul(hy, hx));
        }
        qe = cscale(qe, nb); qc = cscale(qc, nb); qd = cscale(qd, nb); qo = cscale(qo, nb);
        if (fs > 0) {
          add_sp<NS>(ge, fs - 1, qe);
          add_sp<NS>(gd, fs - 1, qd);
          if (GEN) { add_sp<NS>(gc, fs - 1, qc); add_sp<NS>(go, fs - 1, qo); }
          continue;
        }
        for (int sidx = 0; sidx < nk; ++sidx) {
          double m = mt[own + nsm * (kp + nsm * (sidx + (size_t)nsm * kap))];
          if (m == 0.0) continue;
          int sp = spc[sidx + ldspc * kap] - 1;
          add_sp<NS>(ge, sp, cscale(qe, m));
          add_sp<NS>(gd, sp, cscale(qd, m));
          if (GEN) { add_sp<NS>(gc, sp, cscale(qc, m)); add_sp<NS>(go, sp, cscale(qo, m)); }
        }
      }
    }
  }
  // sum over the 32 lanes (one warp = one orbital), fixed order; pa = z e per lane before the sum
  double2 gpa[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    gpa[q] = cmul(z, ge[q]);
    if (!GEN) gc[q] = ge[q];   // o = 0: c enters as e does
  }
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    if (q >= nsp) break;
    for (int off = 16; off > 0; off >>= 1) {
      gc[q].x += __shfl_xor_sync(0xffffffffu, gc[q].x, off);
      gc[q].y += __shfl_xor_sync(0xffffffffu, gc[q].y, off);
      gd[q].x += __shfl_xor_sync(0xffffffffu, gd[q].x, off);
      gd[q].y += __shfl_xor_sync(0xffffffffu, gd[q].y, off);
      gpa[q].x += __shfl_xor_sync(0xffffffffu, gpa[q].x, off);
      gpa[q].y += __shfl_xor_sync(0xffffffffu, gpa[q].y, off);
      go[q].x += __shfl_xor_sync(0xffffffffu, go[q].x, off);
      go[q].y += __shfl_xor_sync(0xffffffffu, go[q].y, off);
      ge[q].x += __shfl_xor_sync(0xffffffffu, ge[q].x, off);
      ge[q].y += __shfl_xor_sync(0xffffffffu, ge[q].y, off);
    }
  }
  if (lane == 0) {
    double2* out = gpart + ((size_t)(tile * gbpt + blk) * NGK) * 9 * nsp;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      if (q >= nsp) break;
      out[(0 * 9 + l) * nsp + q] = gc[q];
      out[(1 * 9 + l) * nsp + q] = gd[q];
      out[(2 * 9 + l) * nsp + q] = gpa[q];
      out[(3 * 9 + l) * nsp + q] = go[q];
      out[(4 * 9 + l) * nsp + q] = ge[q];
    }
  }
}

// k_adj_grad with the register accumulators sized for the operator's species count
template <typename ST, bool GEN, bool WY = false>
void launch_adj_grad(int nsp, unsigned grid, cudaStream_t s, const OpView& ov, const BatchView& bv, const double* mt,
                     const int* spc, int ldspc, const AdjVecs& av, const double2* sk, int gnpb, double2* gpart,
                     const double2* cy = nullptr) {
  if (nsp <= 3)
    k_adj_grad<ST, GEN, WY, 3><<<grid, GPW * TL, 0, s>>>(ov, bv, mt, spc, ldspc, av, sk, gnpb, gpart, cy);
  else if (nsp <= 5)
    k_adj_grad<ST, GEN, WY, 5><<<grid, GPW * TL, 0, s>>>(ov, bv, mt, spc, ldspc, av, sk, gnpb, gpart, cy);
  else
    k_adj_grad<ST, GEN, WY, MAXSP><<<grid, GPW * TL, 0, s>>>(ov, bv, mt, spc, ldspc, av, sk, gnpb, gpart, cy);
}

// gacc[tile][NGK][9][nsp] += sum over the blocks of the step's partials (fixed order)
// grid (ntile, ceil(ng / 32)), RED_THREADS per block: lane j of the block's warps sums entry 32 blockIdx.y + j
__global__ void k_adj_gsum(int ntile, int gbpt, int ng, const int* tile_act, const double2* gpart, double2* gacc) {
  const int tile = blockIdx.x;
  if (tile >= ntile || !tile_act[tile]) return;
  const int e0 = blockIdx.y * TL, e = e0 + threadIdx.x % TL;
  const double2 sum = block_sum_rows(gpart + (size_t)tile * gbpt * ng + e0, gbpt, ng, e < ng);
  if (threadIdx.x < TL && e < ng) gacc[(size_t)tile * ng + e] = cadd(gacc[(size_t)tile * ng + e], sum);
}

// per-lane sum of partials: out[L] = sum_q part[(tile * bpt + q) * TL + lane]
__global__ void k_lane_sum(int ntile, int bpt, const int* tile_act, const double2* part, double2* out) {
  int tile = blockIdx.x;
  if (tile >= ntile) return;
  const double2 sum = tile_act[tile] ? block_sum_rows(part + (size_t)tile * bpt * TL, bpt, TL) : make_double2(0, 0);
  if (threadIdx.x < TL) out[tile * TL + threadIdx.x] = sum;
}

// scalars of reverse step k for every lane (state arrays indexed [lane][NLMAX], k 1-based):
//   phase 0: coefficients of wbar from d1 = ubar_{k+1} . X_{k+1} (raw); with tile_act, a tile takes part in step k
//            when one of its lanes is at least k deep (a warp of the launch is a tile)
//   phase 1: abar', bbar_{k-1} update from d2 = wbar . X_k, d3 = wbar . X_{k-1} (raw), the coefficients of ybar and of
//            ubar_k += A ybar + abar y_k - a_k wbar, ubar_{k-1} -= b_{k-1} wbar
//   phase 2: phase 1 for the fused reverse step, where A ybar = A wbar + abar y_k and ubar_k is written whole:
//            ubar_k = A wbar + 2 abar y_k - a_k wbar - b_k wbar_{k+1} (c5 = 2 abar, c6 = a_k, c4 = b_k below the lane's
//            last level, else 0)
struct AdjScal {
  const double2* a;       // forward a_k
  const double2* b;       // forward b_k
  const int* m;           // depth per lane
  double2* abar;
  double2* bbar;
  double2 *s_next, *s_k, *s_prev;   // scales of X_{k+1}, X_k, X_{k-1}
  double2 *c1, *c2, *c3, *c4, *c5, *c6;
  const double2 *d1, *d2, *d3;
};
__device__ __forceinline__ double2 scale_of(const AdjScal& S, int L, int k) {   // s_k: u_k = s_k X_k
  if (k <= 1) return make_double2(k == 1 ? 1.0 : 0.0, 0.0);
  double2 b = S.b[(size_t)L * NLMAX + k - 2];
  if (cmag(b) == 0.0 || k > S.m[L]) return make_double2(0, 0);
  return cdiv(make_double2(1.0, 0.0), b);
}
__global__ void k_adj_scal(AdjScal S, int nlane, const int* lane_group, int k, int phase, int* tile_act = nullptr) {
  int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlane) return;   // nlane is a multiple of TL: whole warps leave
  if (tile_act) {
    const unsigned any = __ballot_sync(0xffffffffu, lane_group[L] >= 0 && k <= S.m[L]);
    if (L % TL == 0) tile_act[L / TL] = any != 0;
  }
  const double2 zero = make_double2(0, 0);
  if (lane_group[L] < 0 || k > S.m[L]) {
    if (phase == 0) { S.c1[L] = zero; S.c2[L] = zero; S.s_next[L] = zero; S.s_k[L] = zero; S.s_prev[L] = zero; }
    else { S.c3[L] = zero; S.c4[L] = zero; S.c5[L] = zero; S.c6[L] = zero; }
    return;
  }
  const size_t o = (size_t)L * NLMAX;
  if (phase == 0) {
    double2 sn = k < S.m[L] ? scale_of(S, L, k + 1) : zero;
    S.s_next[L] = sn;
    S.s_k[L] = scale_of(S, L, k);
    S.s_prev[L] = scale_of(S, L, k - 1);
    if (k < S.m[L]) {
      double2 bk = S.b[o + k - 1];
      double2 ib = cdiv(make_double2(1.0, 0.0), bk);
      double2 d1 = cmul(sn, S.d1[L]);                           // ubar_{k+1} . u_{k+1}
      double2 bb = csub(S.bbar[o + k - 1], cmul(d1, ib));
      S.bbar[o + k - 1] = bb;
      S.c1[L] = ib;                                              // wbar' = ubar_{k+1} / b_k + bbar_k u_{k+1}
      S.c2[L] = cmul(bb, sn);
    } else {
      S.c1[L] = zero;
      S.c2[L] = zero;
    }
  } else {
    double2 sk = S.s_k[L], sp = S.s_prev[L];
    double2 ab = csub(S.abar[o + k - 1], cmul(sk, S.d2[L]));   // abar_k -= wbar . u_k
    S.abar[o + k - 1] = ab;
    if (k > 1) S.bbar[o + k - 2] = csub(S.bbar[o + k - 2], cmul(sp, S.d3[L]));   // bbar_{k-1} -= wbar . u_{k-1}
    S.c3[L] = cmul(ab, sk);                                      // ybar = wbar + abar u_k
    if (phase == 2) {
      S.c4[L] = k < S.m[L] ? S.b[o + k - 1] : zero;
      S.c5[L] = cscale(ab, 2.0);
    } else {
      S.c4[L] = k > 1 ? S.b[o + k - 2] : zero;                   // ubar_{k-1} -= b_{k-1} wbar
      S.c5[L] = ab;                                              // ubar_k += A ybar + abar y_k - a_k wbar
    }
    S.c6[L] = S.a[o + k - 1];
  }
}

// forward recompute of one level: acur = a_k, bprev = b_{k-1}, su = s_k, sup = s_{k-1}, wact = k < m
__global__ void k_set_fwd(BatchView bv, AdjScal S, int nlane, int k) {
  int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlane) return;
  const size_t o = (size_t)L * NLMAX;
  bool live = bv.lane_group[L] >= 0 && k <= S.m[L];
  bv.acur[L] = live ? S.a[o + k - 1] : make_double2(0, 0);
  bv.bprev[L] = (live && k > 1) ? S.b[o + k - 2] : make_double2(0, 0);
  bv.su[L] = live ? scale_of(S, L, k) : make_double2(0, 0);
  bv.sup[L] = live ? scale_of(S, L, k - 1) : make_double2(0, 0);
  bv.lane_wact[L] = (live && k < S.m[L]) ? 1 : 0;
}

// t2 = S R_d x (unscaled), general or with d folded into the blocks
template <typename ST>
void apply_SD(asr_op* op, const BatchView& bv, bool dunif, const typename St2<ST>::T* x, typename St2<ST>::T* tmp,
              typename St2<ST>::T* t2, double2* part, int npw, int grid, cudaStream_t s) {
  OpView ov = op->view();
  const ST* blk = std::is_same<ST, double>::value ? (const ST*)op->d_blocks : (const ST*)op->d_blocks_f;
  size_t sm = smul_smem(op, sizeof(ST));
  if (dunif) {
    launch_smul<ST, true, false>(op, bv, blk, x, t2, part, npw, grid, s);
  } else {
    k_rand<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, PD, x, tmp, npw);
    launch_smul<ST, false, false>(op, bv, blk, tmp, t2, part, npw, grid, s);
  }
}

// y = s (h x - h O h x + (E + X) x) on the general operator with its intermediates kept: TA = S D x, H = h x, R = O h x,
// TB = S D O h x (unscaled), and the partial dots of the final combination
template <typename ST>
void apply_general_keep(asr_op* op, const BatchView& bv, bool dunif, const typename St2<ST>::T* x, typename St2<ST>::T* y,
                        typename St2<ST>::T* TA, typename St2<ST>::T* H, typename St2<ST>::T* R, typename St2<ST>::T* TB,
                        typename St2<ST>::T* TMP, double2* part, int npw, int grid, cudaStream_t s) {
  OpView ov = op->view();
  apply_SD<ST>(op, bv, dunif, x, TMP, TA, part, npw, grid, s);
  k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, TA, x, PC, false, x, false, nullptr, 1.0, false, H, part, npw);
  k_rand<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, PO, H, R, npw);
  apply_SD<ST>(op, bv, dunif, R, TMP, TB, part, npw, grid, s);
  k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, TB, R, PC, false, x, true, H, -1.0, true, y, part, npw);
}

template <typename ST>
int run_adjoint_t(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                  const GroupLayout& GL, const std::vector<int>& lane_group, const std::vector<double2>& lane_z,
                  const std::vector<double2>& lane_w, double depth_tol, int tail, int project, int stride,
                  std::vector<double2>& g_out, std::vector<int>& m_out, std::vector<double2>& grad_out /* [group][NGK][9][nsp] */) {
  typedef typename St2<ST>::T T2;
  cudaStream_t s = ctx->stream;
  const int nn = op->nn, nsp = op->nsp, nlane = (int)lane_group.size();
  if (nsp > MAXSP) { set_error("adjoint: at most %d species", MAXSP); return ASR_EINVAL; }
  bool dunif = true, gen = false;
  int mmax = 0;
  for (auto& g : ginfo) {
    if (!(g.flags & GF_O_ZERO)) gen = true;   // H = E_nu + h - h o h: the general operator and its intermediates
    if (!(g.flags & GF_D_UNIFORM)) dunif = false;
    mmax = std::max(mmax, g.nlev);
  }
  if (mmax > NLMAX) { set_error("adjoint: depth above %d", NLMAX); return ASR_EINVAL; }
  // Vectors kept for the reverse sweep: every level's (keep = true, no recomputation) when the caller leaves the stride
  // to the library and a batch of at least 4 tiles fits in half the free device memory; else checkpoints every c
  // levels (c = stride, or ceil(sqrt(depth))) with the segments recomputed.  Both give the same G and the same gradient
  // to rounding (bitwise on the operators of the stride tests).
  size_t freeb0 = 0, totb0 = 0;
  cudaMemGetInfo(&freeb0, &totb0);
  freeb0 += ctx->ws_bytes;   // a held slab is this call's to reuse
  const size_t vbytes = (size_t)nn * 9 * TL * sizeof(T2);
  const bool keep = stride <= 0 && (size_t)4 * (3 * mmax + 15 + (gen ? 3 * mmax + 3 : 0)) * vbytes <= freeb0 / 2;
  const int c = keep ? std::max(1, mmax) : std::max(1, stride > 0 ? stride : (int)std::ceil(std::sqrt((double)mmax)));
  const int nseg = (mmax + c - 1) / c;
  // tiles: one group each
  std::vector<std::vector<int>> tiles;
  {
    std::vector<std::vector<int>> per_group(ginfo.size());
    for (int L = 0; L < nlane; ++L) per_group[lane_group[L]].push_back(L);
    for (auto& lst : per_group)
      for (size_t q = 0; q < lst.size(); q += TL)
        tiles.emplace_back(lst.begin() + q, lst.begin() + std::min(lst.size(), q + (size_t)TL));
    // deepest tiles first, so that the tiles of a batch have about one depth: the forward retires a tile at its depth
    // and the reverse sweep skips a tile above it
    std::vector<int> ord(tiles.size()), dep(tiles.size());
    for (size_t t = 0; t < tiles.size(); ++t) { ord[t] = (int)t; dep[t] = ginfo[lane_group[tiles[t][0]]].nlev; }
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return dep[x] > dep[y]; });
    std::vector<std::vector<int>> sorted(tiles.size());
    for (size_t t = 0; t < tiles.size(); ++t) sorted[t] = std::move(tiles[ord[t]]);
    tiles.swap(sorted);
  }
  const int ntile_all = (int)tiles.size();
  // the fused reverse step (o = 0, d uniform): the step kernel applies A to wbar and writes ubar_k in its epilogue
  const bool fusedrev = !gen && dunif;
  // memory: forward 3 + checkpoints 2 nseg + segment (c + 2) X + c Y + c T2 + adjoint 7 (+1 temporary) vectors per tile;
  // the general operator keeps h X, O h X, S D O h X per segment level and h ybar, O h ybar, S D O h ybar (3 c + 3 more)
  const size_t vec_bytes = (size_t)nn * 9 * TL * sizeof(T2);
  const int nvec = 3 + 2 * nseg + (c + 2) + 2 * c + 8 + (gen ? 3 * c + 3 : 0);
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  freeb += ctx->ws_bytes;
  // tiles per batch: as the forward's default (16), halved while the batch's vectors would take more than half the free
  // device memory (a 16-tile batch of the fcc ternary workload holds about 70 GB)
  int tpb = 16;
  if (const char* e = getenv("ASR_TILES_PER_BATCH")) tpb = std::max(1, atoi(e));
  while (tpb > 1 && (size_t)tpb * nvec * vec_bytes > freeb / 2) tpb /= 2;
  if ((size_t)nvec * vec_bytes > freeb) { set_error("adjoint: %d vectors of %zu bytes do not fit", nvec, vec_bytes); return ASR_ENOMEM; }
  tpb = std::min(tpb, ntile_all);
  const int npw = 4, npb = WPB * npw, bpt = (nn + npb - 1) / npb;
  int gnpb = 64;   // nodes per block of the gradient kernel
  if (const char* e = getenv("ASR_ADJ_GRAD_NODES")) gnpb = std::max(1, atoi(e));
  const int gbpt = (nn + gnpb - 1) / gnpb, ngd = NGK * 9 * nsp;
  const int nlp = tpb * TL;
  Dev<double> d_gblob, d_mt;
  Dev<GroupInfo> d_ginfo;
  Dev<int> d_spc;
  ASR_TRY(d_gblob.alloc(gblob.size())); ASR_TRY(d_ginfo.alloc(ginfo.size()));
  ASR_TRY(d_mt.alloc(op->mt.size())); ASR_TRY(d_spc.alloc(op->spc.size()));
  ASR_CUDA(cudaMemcpyAsync(d_gblob.p, gblob.data(), gblob.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_ginfo.p, ginfo.data(), ginfo.size() * sizeof(GroupInfo), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_mt.p, op->mt.data(), op->mt.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_spc.p, op->spc.data(), op->spc.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  Dev<int> d_lgroup, d_act, d_wact, d_m, d_tact, d_tact0, d_nfall, d_tgroup, d_tick;
  Dev<double2> d_a, d_b, d_abar, d_bbar, d_gprev, d_acur, d_bprev, d_su, d_sup, d_part, d_part2, d_z, d_gpart, d_gacc;
  Dev<double2> d_sn, d_sk, d_sp, d_c[6], d_d1, d_d2, d_d3, d_one;
  ASR_TRY(d_lgroup.alloc(nlp)); ASR_TRY(d_act.alloc(nlp)); ASR_TRY(d_wact.alloc(nlp)); ASR_TRY(d_m.alloc(nlp));
  ASR_TRY(d_tact.alloc(tpb)); ASR_TRY(d_tact0.alloc(tpb)); ASR_TRY(d_nfall.alloc(1)); ASR_TRY(d_tgroup.alloc(tpb));
  ASR_TRY(d_tick.alloc(tpb));
  ASR_TRY(d_a.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_b.alloc((size_t)nlp * NLMAX));
  ASR_TRY(d_abar.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_bbar.alloc((size_t)nlp * NLMAX));
  ASR_TRY(d_gprev.alloc(nlp)); ASR_TRY(d_acur.alloc(nlp)); ASR_TRY(d_bprev.alloc(nlp)); ASR_TRY(d_su.alloc(nlp));
  ASR_TRY(d_sup.alloc(nlp)); ASR_TRY(d_part.alloc((size_t)tpb * bpt * TL)); ASR_TRY(d_part2.alloc((size_t)tpb * bpt * TL));
  ASR_TRY(d_z.alloc(nlp)); ASR_TRY(d_gpart.alloc((size_t)tpb * gbpt * ngd)); ASR_TRY(d_gacc.alloc((size_t)tpb * ngd));
  ASR_TRY(d_sn.alloc(nlp)); ASR_TRY(d_sk.alloc(nlp)); ASR_TRY(d_sp.alloc(nlp));
  for (int q = 0; q < 6; ++q) ASR_TRY(d_c[q].alloc(nlp));
  ASR_TRY(d_d1.alloc(nlp)); ASR_TRY(d_d2.alloc(nlp)); ASR_TRY(d_d3.alloc(nlp)); ASR_TRY(d_one.alloc(nlp));
  // the vectors: one slab (the context's held one, or allocated here and freed on return)
  const size_t vlen = (size_t)tpb * nn * 9 * TL;
  Dev<unsigned char> own;
  T2* vbase = nullptr;
  ASR_TRY(vector_slab(ctx, (size_t)nvec * vlen * sizeof(T2), own, (void**)&vbase));
  struct VecRef { T2* p; };
  std::vector<VecRef> V(nvec);
  for (int q = 0; q < nvec; ++q) V[q].p = vbase + (size_t)q * vlen;
  T2* FW[3] = {V[0].p, V[1].p, V[2].p};
  auto CK = [&](int j, int which) { return V[3 + 2 * j + which].p; };          // checkpoint j: X_{k0-1}, X_{k0}
  const int xs0 = 3 + 2 * nseg;
  auto XS = [&](int q) { return V[xs0 + q].p; };                               // X_{k0-1+q}, q = 0 .. c+1
  auto YS = [&](int q) { return V[xs0 + c + 2 + q].p; };
  auto TS = [&](int q) { return V[xs0 + 2 * c + 2 + q].p; };
  const int ab0 = xs0 + 3 * c + 2;
  T2* UB[3] = {V[ab0].p, V[ab0 + 1].p, V[ab0 + 2].p};
  T2* WB = V[ab0 + 3].p;
  T2* YB = V[ab0 + 4].p;
  T2* T2B = V[ab0 + 5].p;
  T2* AY = V[ab0 + 6].p;
  T2* TMP = V[ab0 + 7].p;
  const int gs0 = ab0 + 8;   // general operator: per segment level q the intermediates of X, then those of ybar
  auto HS = [&](int q) { return gen ? V[gs0 + q].p : nullptr; };
  auto RS = [&](int q) { return gen ? V[gs0 + c + q].p : nullptr; };
  auto QS = [&](int q) { return gen ? V[gs0 + 2 * c + q].p : nullptr; };
  T2* HB = gen ? V[gs0 + 3 * c].p : nullptr;
  T2* RB = gen ? V[gs0 + 3 * c + 1].p : nullptr;
  T2* QB = gen ? V[gs0 + 3 * c + 2].p : nullptr;
  g_out.assign(nlane, make_double2(0, 0));
  m_out.assign(nlane, 0);
  grad_out.assign(ginfo.size() * (size_t)ngd, make_double2(0, 0));
  std::vector<double2> ones(nlp, make_double2(1.0, 0.0));
  ASR_CUDA(cudaMemcpyAsync(d_one.p, ones.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
  std::vector<int> hgroup(nlp), lmap(nlp), hm(nlp);
  std::vector<double2> hz(nlp), ha((size_t)nlp * NLMAX), hb((size_t)nlp * NLMAX), habar((size_t)nlp * NLMAX), hbbar((size_t)nlp * NLMAX);
  std::vector<double2> hgacc((size_t)tpb * ngd);
  OpView ov = op->view();
  const ST* blk = std::is_same<ST, double>::value ? (const ST*)op->d_blocks : (const ST*)op->d_blocks_f;
  for (int t0 = 0; t0 < ntile_all; t0 += tpb) {
    NvtxRange batch_range("adjoint batch");
    NvtxPhase phase;
    phase.next("adjoint forward");
    const int nt = std::min(tpb, ntile_all - t0);
    std::vector<int> tact(tpb, 0), act(nlp, 0), tgroup(tpb, -1);
    for (int q = 0; q < nlp; ++q) {
      int bt = q / TL, L = -1;
      if (bt < nt && q % TL < (int)tiles[t0 + bt].size()) L = tiles[t0 + bt][q % TL];
      lmap[q] = L;
      hgroup[q] = L >= 0 ? lane_group[L] : -1;
      hz[q] = L >= 0 ? lane_z[L] : make_double2(0, 0);
      if (L >= 0) { tact[bt] = 1; act[q] = 1; tgroup[bt] = hgroup[q]; }
    }
    ASR_CUDA(cudaMemcpyAsync(d_lgroup.p, hgroup.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tgroup.p, tgroup.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_act.p, act.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tact.p, tact.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tact0.p, d_tact.p, tpb * sizeof(int), cudaMemcpyDeviceToDevice, s));
    ASR_CUDA(cudaMemsetAsync(d_tick.p, 0, tpb * sizeof(int), s));
    ASR_CUDA(cudaMemcpyAsync(d_z.p, hz.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_su.p, ones.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemsetAsync(d_wact.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_m.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_a.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_b.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_gprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_bprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_sup.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_nfall.p, 0, sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_gacc.p, 0, (size_t)tpb * ngd * sizeof(double2), s));
    // the forward stops each lane by the depth test of src/asr_edc.f90:121-127 when depth_tol > 0; the reverse sweep then
    // differentiates the chain at the depth it stopped at
    BatchView bv{nt, nn, op->nsmax, 0, ASR_MODE_EDC, project, tail, NLMAX, depth_tol, d_gblob.p, GL, d_ginfo.p, d_lgroup.p,
                 d_tgroup.p, d_z.p, d_act.p, d_wact.p, d_m.p, d_a.p, d_b.p, d_gprev.p, d_acur.p, d_bprev.p, d_su.p, d_sup.p,
                 d_tact.p, d_nfall.p};
    const int grid = nt * bpt;
    int kmax = 0;
    for (int q = 0; q < nlp; ++q) if (hgroup[q] >= 0) kmax = std::max(kmax, ginfo[hgroup[q]].nlev);
    // ---- forward with checkpoints (X_{k0-1}, X_{k0}) at k0 = 1 + j c, or keeping every level in the segment buffers.
    // The Lanczos update reduces b_k in its epilogue (the tile's last block), the fused step a_k except at the levels of
    // the depth test, whose fraction evaluation runs in the separate reduction kernel: the sums are those of the separate
    // kernels, in the same order.
    auto depth_due = [&](int k) { return depth_tol > 0.0 && k >= 8 && k % 4 == 0; };
    // algorithmic work of the forward's kernels (the step's vector streams: read U, write Y, and t2 where kept; the node
    // tables per tile), as the forward chains count them
    const double tab = (double)op->nslot * 5 + (double)op->nsmax * 5 + 8 + 8 + 4;
    auto step_bytes = [&](int streams) { return (double)nt * nn * (streams * 9.0 * TL * sizeof(T2) + tab); };
    const double step_flops = (double)nt * nn * TL * (op->nslot + 1) * 81.0 * 4.0;
    const double lanczos_bytes = (double)nt * nn * 4.0 * 9 * TL * sizeof(T2), lanczos_flops = (double)nt * nn * TL * 9 * 30.0;
    const double vstream = (double)nt * nn * 9 * TL * sizeof(T2), sflops = step_flops;   // one vector stream; one S application
    const size_t cpy = (size_t)nt * nn * 9 * TL * sizeof(T2);
    if (keep) {
      k_init<ST><<<std::min<size_t>(65535, ((size_t)nt * nn * 9 * TL + 255) / 256), 256, 0, s>>>(bv, XS(1), XS(0));
      for (int k = 1; k <= kmax; ++k) {   // the recomputation's step, with the reductions of the forward
        const int q = k - 1;
        const bool a_in_step = fusedrev && !depth_due(k);
        int ps = ctx->prof_start(s);
        if (gen) {
          apply_general_keep<ST>(op, bv, dunif, XS(q + 1), YS(q), TS(q), HS(q), RS(q), QS(q), TMP, d_part.p, npw, grid, s);
        } else if (dunif) {
          BatchView bvt = bv;
          bvt.kstep = k;
          bvt.t2out = TS(q);
          bvt.tick = a_in_step ? d_tick.p : nullptr;
          launch_smul<ST, true, true, 1>(op, bvt, blk, XS(q + 1), YS(q), d_part.p, npw, grid, s);
        } else {
          apply_SD<ST>(op, bv, dunif, XS(q + 1), TMP, TS(q), d_part.p, npw, grid, s);
          k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, TS(q), XS(q + 1), PCEB, true, XS(q + 1), false, nullptr, 1.0, true,
                                                  YS(q), d_part.p, npw);
        }
        ctx->prof_stop(s, ps, ASR_KERNEL_STEP, step_bytes(3), step_flops);
        if (!a_in_step) k_reduce_a<<<nt, RED_THREADS, 0, s>>>(bv, d_part.p, bpt, k);
        BatchView bvw = bv;
        bvw.kstep = k;
        bvw.tick = d_tick.p;
        ps = ctx->prof_start(s);
        k_lanczos_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bvw, YS(q), XS(q + 1), XS(q), d_part.p, npw, XS(q + 2));
        ctx->prof_stop(s, ps, ASR_KERNEL_LANCZOS, lanczos_bytes, lanczos_flops);
      }
    } else {
      k_init<ST><<<std::min<size_t>(65535, ((size_t)nt * nn * 9 * TL + 255) / 256), 256, 0, s>>>(bv, FW[1], FW[0]);
      ASR_CUDA(cudaMemcpyAsync(CK(0, 0), FW[0], cpy, cudaMemcpyDeviceToDevice, s));
      ASR_CUDA(cudaMemcpyAsync(CK(0, 1), FW[1], cpy, cudaMemcpyDeviceToDevice, s));
    }
    for (int k = 1; k <= (keep ? 0 : kmax); ++k) {
      T2* U = FW[k % 3];
      T2* UP = FW[(k + 2) % 3];
      T2* Y = FW[(k + 1) % 3];
      const bool a_in_step = fusedrev && !depth_due(k);
      int ps = ctx->prof_start(s);
      if (gen) {
        apply_general_keep<ST>(op, bv, dunif, U, Y, AY, WB, YB, T2B, TMP, d_part.p, npw, grid, s);
      } else if (dunif) {   // the fused step of the forward chains (d folded into the blocks)
        BatchView bvt = bv;
        bvt.kstep = k;
        bvt.tick = a_in_step ? d_tick.p : nullptr;
        launch_smul<ST, true, true>(op, bvt, blk, U, Y, d_part.p, npw, grid, s);
      } else {
        apply_SD<ST>(op, bv, dunif, U, TMP, AY, d_part.p, npw, grid, s);
        k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, AY, U, PCEB, true, U, false, nullptr, 1.0, true, Y, d_part.p, npw);
      }
      ctx->prof_stop(s, ps, ASR_KERNEL_STEP, step_bytes(2), step_flops);
      if (!a_in_step) k_reduce_a<<<nt, RED_THREADS, 0, s>>>(bv, d_part.p, bpt, k);
      BatchView bvw = bv;
      bvw.kstep = k;
      bvw.tick = d_tick.p;
      ps = ctx->prof_start(s);
      k_lanczos_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bvw, Y, U, UP, d_part.p, npw);
      ctx->prof_stop(s, ps, ASR_KERNEL_LANCZOS, lanczos_bytes, lanczos_flops);
      if (k % c == 0 && k / c < nseg) {   // X_k and X_{k+1} start segment k / c
        ASR_CUDA(cudaMemcpyAsync(CK(k / c, 0), U, cpy, cudaMemcpyDeviceToDevice, s));
        ASR_CUDA(cudaMemcpyAsync(CK(k / c, 1), Y, cpy, cudaMemcpyDeviceToDevice, s));
      }
    }
    ASR_CUDA(cudaGetLastError());
    // the forward retired finished tiles; the recomputation visits every tile of the batch, the reverse step k the tiles
    // with a lane at least k deep (k_adj_scal)
    ASR_CUDA(cudaMemcpyAsync(d_tact.p, d_tact0.p, tpb * sizeof(int), cudaMemcpyDeviceToDevice, s));
    phase.next("fraction adjoint (host)");
    // ---- fraction adjoint on the host: G and the seeds abar, bbar
    ASR_CUDA(cudaMemcpyAsync(hm.data(), d_m.p, nlp * sizeof(int), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaMemcpyAsync(ha.data(), d_a.p, ha.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaMemcpyAsync(hb.data(), d_b.p, hb.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    std::fill(habar.begin(), habar.end(), make_double2(0, 0));
    std::fill(hbbar.begin(), hbbar.end(), make_double2(0, 0));
    {
      std::vector<double2> w1(NLMAX), w2(NLMAX), w3(NLMAX), w4(NLMAX), w5(NLMAX);
      for (int q = 0; q < nlp; ++q) {
        int L = lmap[q];
        if (L < 0 || hm[q] < 1) continue;
        m_out[L] = hm[q];
        g_out[L] = cf_species_adjoint(&ha[(size_t)q * NLMAX], &hb[(size_t)q * NLMAX], hm[q], lane_z[L], tail, lane_w[L],
                                      &habar[(size_t)q * NLMAX], &hbbar[(size_t)q * NLMAX], w1.data(), w2.data(), w3.data(),
                                      w4.data(), w5.data());
      }
    }
    ASR_CUDA(cudaMemcpyAsync(d_abar.p, habar.data(), habar.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_bbar.p, hbbar.data(), hbbar.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
    AdjScal S{d_a.p, d_b.p, d_m.p, d_abar.p, d_bbar.p, d_sn.p, d_sk.p, d_sp.p, d_c[0].p, d_c[1].p, d_c[2].p, d_c[3].p, d_c[4].p,
              d_c[5].p, d_d1.p, d_d2.p, d_d3.p};
    // adjoint BatchView: unit scales for applying A to ybar
    BatchView bva = bv;
    bva.su = d_one.p;
    // ubar (three rotating buffers; two in the fused step, which writes ubar_k whole) and, in the fused step, wbar of
    // this and the previous level (WB, YB alternating) start at zero; d1 = ubar_{k+1} . X_{k+1} is zero above the top
    for (int q = 0; q < 3; ++q) ASR_CUDA(cudaMemsetAsync(UB[q], 0, cpy, s));
    if (fusedrev) {
      ASR_CUDA(cudaMemsetAsync(WB, 0, cpy, s));
      ASR_CUDA(cudaMemsetAsync(YB, 0, cpy, s));
      ASR_CUDA(cudaMemsetAsync(d_d1.p, 0, nlp * sizeof(double2), s));
    }
    T2* WBF[2] = {WB, YB};
    phase.next("adjoint reverse");
    for (int j = nseg - 1; j >= 0; --j) {
      const int k0 = 1 + j * c, k1 = std::min(kmax, k0 + c - 1);
      if (k0 > kmax) continue;
      // recompute X_{k0-1} .. X_{k1+1}, Y_k, T2_k (kept from the forward in the keep mode) on every tile of the batch
      if (!keep) {
        ASR_CUDA(cudaMemcpyAsync(d_tact.p, d_tact0.p, tpb * sizeof(int), cudaMemcpyDeviceToDevice, s));
        ASR_CUDA(cudaMemcpyAsync(XS(0), CK(j, 0), cpy, cudaMemcpyDeviceToDevice, s));
        ASR_CUDA(cudaMemcpyAsync(XS(1), CK(j, 1), cpy, cudaMemcpyDeviceToDevice, s));
      }
      for (int k = k0; k <= (keep ? k0 - 1 : k1); ++k) {
        int q = k - k0;
        k_set_fwd<<<(nlp + 127) / 128, 128, 0, s>>>(bv, S, nlp, k);
        if (gen) {
          apply_general_keep<ST>(op, bv, dunif, XS(q + 1), YS(q), TS(q), HS(q), RS(q), QS(q), TMP, d_part.p, npw, grid, s);
        } else if (dunif) {   // the forward's fused step, bit for bit, with t2 = S d X stored for the gradient
          BatchView bvt = bv;
          bvt.t2out = TS(q);
          launch_smul<ST, true, true, 1>(op, bvt, blk, XS(q + 1), YS(q), d_part.p, npw, grid, s);
        } else {
          apply_SD<ST>(op, bv, dunif, XS(q + 1), TMP, TS(q), d_part.p, npw, grid, s);
          k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, TS(q), XS(q + 1), PCEB, true, XS(q + 1), false, nullptr, 1.0, true,
                                                  YS(q), d_part.p, npw);
        }
        k_lanczos_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, YS(q), XS(q + 1), XS(q), d_part.p, npw, XS(q + 2));
      }
      // reverse k = k1 .. k0
      for (int k = k1; k >= k0 && fusedrev; --k) {
        // wbar_k = P (ubar_{k+1} / b_k + bbar_k u_{k+1}); then one step kernel on wbar_k (unit scales) gives S D wbar_k
        // and, by linearity (A ybar = A wbar + abar y_k), ubar_k = A wbar_k + 2 abar y_k - a_k wbar_k - b_k wbar_{k+1}
        // with the dots ubar_k . X_k of the next step; the gradient kernel forms ybar = wbar + abar u_k and
        // S D ybar = S D wbar + abar S D u_k itself
        const int q = k - k0;
        T2* wk = WBF[k % 2];
        T2* wn = WBF[(k + 1) % 2];
        T2* ubk = UB[k % 2];
        T2* ubn = UB[(k + 1) % 2];
        const int ps = ctx->prof_start(s);
        int pp = ctx->prof_start(s);
        k_adj_scal<<<(nlp + 127) / 128, 128, 0, s>>>(S, nlp, d_lgroup.p, k, 0, d_tact.p);
        ctx->prof_stop(s, pp, ASR_KERNEL_ADJ_SCAL, 0.0, 0.0);
        pp = ctx->prof_start(s);
        k_adj_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bva, ubn, XS(q + 2), XS(q + 1), XS(q), d_c[0].p, d_c[1].p, wk, d_part.p, d_part2.p,
                                              npw);
        ctx->prof_stop(s, pp, ASR_KERNEL_ADJ_VEC, vstream * 5.0, 0.0);
        pp = ctx->prof_start(s);
        k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part.p, d_d2.p);
        k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part2.p, d_d3.p);
        k_adj_scal<<<(nlp + 127) / 128, 128, 0, s>>>(S, nlp, d_lgroup.p, k, 2);
        ctx->prof_stop(s, pp, ASR_KERNEL_ADJ_SCAL, 0.0, 0.0);
        BatchView bvt = bva;
        bvt.t2out = T2B;
        bvt.adj = AdjEpi{YS(q), wn, XS(q + 1), ubk, d_c[4].p, d_c[5].p, d_c[3].p};
        pp = ctx->prof_start(s);
        launch_smul<ST, true, true, 2>(op, bvt, blk, wk, nullptr, d_part.p, npw, grid, s);
        ctx->prof_stop(s, pp, ASR_KERNEL_ADJ_STEP, vstream * 6.0, sflops);
        pp = ctx->prof_start(s);
        k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part.p, d_d1.p);
        ctx->prof_stop(s, pp, ASR_KERNEL_ADJ_SCAL, 0.0, 0.0);
        AdjVecs av{wk, T2B, nullptr, nullptr, nullptr, XS(q + 1), TS(q), nullptr, nullptr, nullptr};
        pp = ctx->prof_start(s);
        launch_adj_grad<ST, false, true>(nsp, nt * gbpt, s, ov, bva, d_mt.p, d_spc.p, op->ldspc, av, d_sk.p, gnpb, d_gpart.p,
                                         d_c[2].p);
        k_adj_gsum<<<dim3(nt, (ngd + TL - 1) / TL), RED_THREADS, 0, s>>>(nt, gbpt, ngd, d_tact.p, d_gpart.p, d_gacc.p);
        ctx->prof_stop(s, pp, ASR_KERNEL_ADJ_GRAD, vstream * 4.0, 0.0);
        // one fused reverse level: 15 vector streams per (node, lane) (w-bar 5, step 6, parameter gradient 4); flops of its
        // one S application
        ctx->prof_stop(s, ps, ASR_KERNEL_ADJOINT, vstream * 15.0, sflops);
      }
      for (int k = k1; k >= k0 && !fusedrev; --k) {
        int q = k - k0;
        T2* ubn = UB[(k + 1) % 3];
        T2* ubk = UB[k % 3];
        T2* ubp = UB[(k + 2) % 3];
        const int ps = ctx->prof_start(s);
        k_dot<ST><<<grid, WPB * TL, 0, s>>>(ov, bva, ubn, XS(q + 2), d_part.p, npw);
        k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part.p, d_d1.p);
        k_adj_scal<<<(nlp + 127) / 128, 128, 0, s>>>(S, nlp, d_lgroup.p, k, 0, d_tact.p);
        k_adj_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bva, ubn, XS(q + 2), XS(q + 1), XS(q), d_c[0].p, d_c[1].p, WB, d_part.p, d_part2.p,
                                              npw);
        k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part.p, d_d2.p);
        k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part2.p, d_d3.p);
        k_adj_scal<<<(nlp + 127) / 128, 128, 0, s>>>(S, nlp, d_lgroup.p, k, 1);
        k_adj_y<ST><<<grid, WPB * TL, 0, s>>>(ov, bva, WB, XS(q + 1), d_c[2].p, d_c[3].p, YB, k > 1 ? ubp : nullptr, npw);
        // A ybar (unit scale) and t2bar = S R_d ybar (the general operator: also h ybar, O h ybar, S D O h ybar)
        if (gen) {
          apply_general_keep<ST>(op, bva, dunif, YB, AY, T2B, HB, RB, QB, TMP, d_part.p, npw, grid, s);
        } else if (dunif) {
          BatchView bvt = bva;
          bvt.t2out = T2B;
          launch_smul<ST, true, true, 1>(op, bvt, blk, YB, AY, d_part.p, npw, grid, s);
        } else {
          apply_SD<ST>(op, bva, dunif, YB, TMP, T2B, d_part.p, npw, grid, s);
          k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bva, T2B, YB, PCEB, true, YB, false, nullptr, 1.0, true, AY, d_part.p, npw);
        }
        k_adj_u<ST><<<grid, WPB * TL, 0, s>>>(ov, bva, AY, YS(q), WB, d_c[4].p, d_c[5].p, ubk, npw);
        AdjVecs av{YB, T2B, HB, RB, QB, XS(q + 1), TS(q), HS(q), RS(q), QS(q)};
        if (gen)
          launch_adj_grad<ST, true>(nsp, nt * gbpt, s, ov, bva, d_mt.p, d_spc.p, op->ldspc, av, d_sk.p, gnpb, d_gpart.p);
        else
          launch_adj_grad<ST, false>(nsp, nt * gbpt, s, ov, bva, d_mt.p, d_spc.p, op->ldspc, av, d_sk.p, gnpb, d_gpart.p);
        k_adj_gsum<<<dim3(nt, (ngd + TL - 1) / TL), RED_THREADS, 0, s>>>(nt, gbpt, ngd, d_tact.p, d_gpart.p, d_gacc.p);
        ASR_CUDA(cudaMemsetAsync(ubn, 0, cpy, s));   // becomes ubar_{k-2}
        // one reverse level: 26 vector streams per (node, lane) over its kernels (dot 2, w-bar 5, y-bar 4, S application
        // 2, combine 3, u-bar 5, parameter gradient 4, clear 1); flops of its one S application
        ctx->prof_stop(s, ps, ASR_KERNEL_ADJOINT, (double)nt * nn * 26.0 * 9 * TL * sizeof(T2),
                       (double)nt * nn * TL * (op->nslot + 1) * 81.0 * 4.0);
      }
    }
    ASR_CUDA(cudaGetLastError());
    ASR_CUDA(cudaMemcpyAsync(hgacc.data(), d_gacc.p, (size_t)tpb * ngd * sizeof(double2), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    ASR_CUDA(cudaGetLastError());
    for (int bt = 0; bt < nt; ++bt) {
      int gq = tgroup[bt];
      if (gq < 0) continue;
      for (int e = 0; e < ngd; ++e) grad_out[(size_t)gq * ngd + e] = cadd(grad_out[(size_t)gq * ngd + e], hgacc[(size_t)bt * ngd + e]);
    }
    // launches per level: forward (operator, a reduction unless in the step, Lanczos update), recomputation (scalars,
    // operator, update), reverse (fused: 9; else 11 and the operator); the depth test's separate reductions not counted
    const int nsd = dunif ? 1 : 2;                                       // one S application
    const int nap = gen ? 2 * nsd + 3 : (dunif ? 1 : nsd + 1);           // one operator application
    const int fwd = fusedrev ? 2 : nap + 2, rev = fusedrev ? 9 : nap + 11;
    ctx->launches += 1 + (int64_t)kmax * (fwd + (keep ? 0 : nap + 2) + rev);
  }
  ASR_TRY(check_wait_error(ctx));
  return ASR_OK;
}

// ================================================================================================ route ed3
// src/asr_ed3.f90: chains on H_eff = z - K'(z), K' = et - h' + u h' + h' u - h' Qt h', h' = g + d S d, with
// et = z ea + eb, u = z ua + ub, Qt = z qa + qb per (orbital, species) in the blob slots
//   PC = g, PD = d, PO = ea, PE = eb, PA = ua, PB = ub, PCEB = qa, PEB = qb.
// Two chains per (group, energy): kind 0 from |a>/|a| with projection vector |v>, kind 1 from |v>/|v| with |a>, where
// |v> = h'|e> (projected) and |a> = |e> + o_c |v>.  Lanes L = 2 (group-energy index) + kind.
enum { E3_G = PC, E3_D = PD, E3_EA = PO, E3_EB = PE, E3_UA = PA, E3_UB = PB, E3_QA = PCEB, E3_QB = PEB };

// T3 = R_u(U) - R_Qt(T1)
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_ed3_t3(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ U,
                                                     const typename St2<ST>::T* __restrict__ T1, typename St2<ST>::T* __restrict__ T3,
                                                     int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = bv.lane_group[L];
  if (grp < 0) return;
  const GroupInfo gi = bv.ginfo[grp];
  const double* gb = bv.gblob + (size_t)grp * bv.GL.stride;
  const double2 z = bv.lane_z[L];
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    double2 xu[9], xt[9], o1[9], o2[9];
    for (int l = 0; l < 9; ++l) {
      size_t q = vix(it.tile, bv.nn, i, l) + lane;
      xu[l] = ld(U + q);
      xt[l] = ld(T1 + q);
    }
    rand_term(op, gi, gb, bv.GL, E3_UB, E3_UA, z, U, it.tile, i, lane, o1, xu);
    rand_term(op, gi, gb, bv.GL, E3_QB, E3_QA, z, T1, it.tile, i, lane, o2, xt);
    for (int l = 0; l < 9; ++l) stv(T3 + vix(it.tile, bv.nn, i, l) + lane, csub(o1[l], o2[l]));
  }
}

// Y = s (z U - K'U) with K'U = R_et(U) - T1 + R_u(T1) + h'(T3), h'(T3) = R_g(T3) + d o T3a (T3a = S d T3); partials
// a = sum norb (s U) . Y and c = sum norb TV . (s U)
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_ed3_w(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ U,
                                                    const typename St2<ST>::T* __restrict__ T1,
                                                    const typename St2<ST>::T* __restrict__ T3,
                                                    const typename St2<ST>::T* __restrict__ T3a,
                                                    const typename St2<ST>::T* __restrict__ TV, typename St2<ST>::T* __restrict__ Y,
                                                    double2* part_a, double2* part_c, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = bv.lane_group[L];
  double2 da = make_double2(0, 0), dc = make_double2(0, 0);
  if (grp >= 0) {
    const GroupInfo gi = bv.ginfo[grp];
    const double* gb = bv.gblob + (size_t)grp * bv.GL.stride;
    const double2 z = bv.lane_z[L], s = bv.su[L];
    for (int qn = 0; qn < npw; ++qn) {
      int i = it.first + w + WPB * qn;
      if (i >= bv.nn) break;
      double2 xu[9], xt1[9], xt3[9], r1[9], r2[9], r3[9], r4[9];
      for (int l = 0; l < 9; ++l) {
        size_t q = vix(it.tile, bv.nn, i, l) + lane;
        xu[l] = ld(U + q);
        xt1[l] = ld(T1 + q);
        xt3[l] = ld(T3 + q);
      }
      rand_term(op, gi, gb, bv.GL, E3_EB, E3_EA, z, U, it.tile, i, lane, r1, xu);     // et U
      rand_term(op, gi, gb, bv.GL, E3_UB, E3_UA, z, T1, it.tile, i, lane, r2, xt1);   // u T1
      rand_term(op, gi, gb, bv.GL, E3_G, -1, z, T3, it.tile, i, lane, r3, xt3);       // g T3
      if (gi.flags & GF_D_UNIFORM) {
        for (int l = 0; l < 9; ++l) r4[l] = cscale(ld(T3a + vix(it.tile, bv.nn, i, l) + lane), gi.dd[l]);
      } else {
        double2 xa[9];
        for (int l = 0; l < 9; ++l) xa[l] = ld(T3a + vix(it.tile, bv.nn, i, l) + lane);
        rand_term(op, gi, gb, bv.GL, E3_D, -1, z, T3a, it.tile, i, lane, r4, xa);
      }
      const double norb = op.sq[i] * op.sq[i];
      double2 en = make_double2(0, 0), ec = make_double2(0, 0);
      for (int l = 0; l < 9; ++l) {
        size_t q = vix(it.tile, bv.nn, i, l) + lane;
        double2 kx = cadd(csub(r1[l], xt1[l]), cadd(r2[l], cadd(r3[l], r4[l])));
        double2 y = cmul(s, csub(cmul(z, xu[l]), kx));
        stv(Y + q, y);
        double2 su_ = cmul(s, xu[l]);
        en = cadd(en, cmul(su_, y));
        ec = cadd(ec, cmul(ld(TV + q), su_));
      }
      da = cadd(da, cscale(en, norb));
      dc = cadd(dc, cscale(ec, norb));
    }
  }
  block_reduce_store(da, part_a, it.tile, bpt);
  __syncthreads();
  block_reduce_store(dc, part_c, it.tile, bpt);
}

// a_k, c_k and the depth test of src/asr_ed3.f90:173-179 (g and the projection f)
__global__ void k_ed3_reduce_a(BatchView bv, const double2* part_a, const double2* part_c, int bpt, int k, double2* ccoef,
                               double2* fprev, const double* tnorm) {
  int tile = blockIdx.x, lane = threadIdx.x;
  if (tile >= bv.ntile || !bv.tile_act[tile]) return;
  const double2 a = block_sum_rows(part_a + (size_t)tile * bpt * TL, bpt, TL);
  const double2 c = block_sum_rows(part_c + (size_t)tile * bpt * TL, bpt, TL);
  if (lane >= TL) return;
  int L = tile * TL + lane;
  int grp = bv.lane_group[L];
  bv.lane_wact[L] = 0;
  if (grp < 0 || !bv.lane_act[L]) return;
  bv.acur[L] = a;
  bv.acoef[(size_t)L * NLMAX + k - 1] = a;
  ccoef[(size_t)L * NLMAX + k - 1] = c;
  bv.lane_m[L] = k;
  int nlev = bv.ginfo[grp].nlev;
  bool go = k < nlev;
  if (go && bv.depth_tol > 0.0 && k >= 8 && k % 4 == 0) {
    double2 gt[NLMAX], wd[NLMAX], we[NLMAX], f;
    int nf = 0;
    double2 g = cf_species_f_dev(bv.acoef + (size_t)L * NLMAX, bv.bcoef + (size_t)L * NLMAX, ccoef + (size_t)L * NLMAX, k,
                                 bv.lane_z[L], bv.tail, false, gt, wd, we, &nf, f);
    if (nf) atomicAdd(bv.nfall, nf);
    if (k > 8) {
      double ag = cmag(g), af = cmag(f);
      if (cmag(csub(g, bv.gprev[L])) <= bv.depth_tol * ag && cmag(csub(f, fprev[L])) <= bv.depth_tol * fmax(af, tnorm[L] * ag))
        go = false;
    }
    bv.gprev[L] = g;
    fprev[L] = f;
  }
  if (go) bv.lane_wact[L] = 1;
  else bv.lane_act[L] = 0;
}

// |v>.|v> and |a>.|a> (|a> = |e> + o_c |v>, |e> the start orbital at node 0) per lane: two partial arrays
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_ed3_dots(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ VV,
                                                       const double* oc, double2* part_v, double2* part_a, int npw) {
  NodeIter it;
  int bpt;
  if (!node_iter(bv, npw, it, bpt)) return;
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = bv.lane_group[L];
  double2 dv = make_double2(0, 0), da = make_double2(0, 0);
  if (grp >= 0) {
    const int l0 = bv.ginfo[grp].l0 - 1;
    const double o = oc[grp];
    for (int qn = 0; qn < npw; ++qn) {
      int i = it.first + w + WPB * qn;
      if (i >= bv.nn) break;
      double2 ev = make_double2(0, 0), ea = make_double2(0, 0);
      for (int l = 0; l < 9; ++l) {
        double2 v = ld(VV + vix(it.tile, bv.nn, i, l) + lane);
        double2 a = cscale(v, o);
        if (i == 0 && l == l0) a.x += 1.0;
        ev = cadd(ev, cmul(v, v));
        ea = cadd(ea, cmul(a, a));
      }
      double nb = op.sq[i] * op.sq[i];
      dv = cadd(dv, cscale(ev, nb));
      da = cadd(da, cscale(ea, nb));
    }
  }
  block_reduce_store(dv, part_v, it.tile, bpt);
  __syncthreads();
  block_reduce_store(da, part_a, it.tile, bpt);
}

// start vectors: kind 0: U = |a> / na, TV = |v>; kind 1: U = |v> / nv, TV = |a>; UP = 0
template <typename ST>
__global__ void k_ed3_start(BatchView bv, const typename St2<ST>::T* __restrict__ VV, const double* oc, const int* kind,
                            const double* na, const double* nv, typename St2<ST>::T* U, typename St2<ST>::T* UP,
                            typename St2<ST>::T* TV) {
  size_t n = (size_t)bv.ntile * bv.nn * 9 * TL;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int lane = (int)(q % TL);
    size_t rest = q / TL;
    int l = (int)(rest % 9);
    size_t nt = rest / 9;
    int node = (int)(nt % bv.nn);
    int tile = (int)(nt / bv.nn);
    int L = tile * TL + lane;
    int grp = bv.lane_group[L];
    double2 u = make_double2(0, 0), t = make_double2(0, 0);
    if (grp >= 0) {
      double2 v = ld(VV + q);
      double2 a = cscale(v, oc[grp]);
      if (node == 0 && l == bv.ginfo[grp].l0 - 1) a.x += 1.0;
      if (kind[L] == 0) { u = cscale(a, 1.0 / na[L]); t = v; }
      else { u = cscale(v, 1.0 / nv[L]); t = a; }
    }
    stv(U + q, u);
    stv(UP + q, make_double2(0, 0));
    stv(TV + q, t);
  }
}

// final fractions of every lane: g and the projection f (cf_species or, for a closed chain, cf_closed)
__global__ void k_ed3_final(BatchView bv, int nlane, const int* lmap, const double2* ccoef, const int* closed, double2* g,
                            double2* f) {
  int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlane) return;
  int dst = lmap[L];
  if (bv.lane_group[L] < 0 || dst < 0) return;
  int m = bv.lane_m[L];
  double2 gt[NLMAX], wd[NLMAX], we[NLMAX], ff = make_double2(0, 0), gg = make_double2(0, 0);
  int nf = 0;
  if (m > 0)
    gg = cf_species_f_dev(bv.acoef + (size_t)L * NLMAX, bv.bcoef + (size_t)L * NLMAX, ccoef + (size_t)L * NLMAX, m, bv.lane_z[L],
                          bv.tail, closed[L] != 0, gt, wd, we, &nf, ff);
  if (nf) atomicAdd(bv.nfall, nf);
  g[dst] = gg;
  f[dst] = ff;
}

template <typename ST>
int run_ed3_t(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
              const GroupLayout& GL, const std::vector<double>& oc, const std::vector<int>& lane_group,
              const std::vector<int>& lane_kind, const std::vector<double2>& lane_z, double depth_tol, int tail, int project,
              std::vector<double2>& g_out, std::vector<double2>& f_out, std::vector<double>& na_out, std::vector<double>& nv_out,
              std::vector<int>& m_out, std::vector<double2>* a_out, std::vector<double2>* b_out, std::vector<double2>* c_out,
              int64_t* nfall_out) {
  typedef typename St2<ST>::T T2;
  cudaStream_t s = ctx->stream;
  const int nn = op->nn, nlane = (int)lane_group.size();
  bool dunif = true;
  for (auto& g : ginfo) {
    if (!(g.flags & GF_D_UNIFORM)) dunif = false;
    if (g.nlev > NLMAX) { set_error("ed3: depth %d above %d", g.nlev, NLMAX); return ASR_EINVAL; }
  }
  std::vector<std::vector<int>> tiles;
  {
    std::vector<std::vector<int>> per_group(ginfo.size());
    for (int L = 0; L < nlane; ++L) per_group[lane_group[L]].push_back(L);
    for (auto& lst : per_group)
      for (size_t q = 0; q < lst.size(); q += TL)
        tiles.emplace_back(lst.begin() + q, lst.begin() + std::min(lst.size(), q + (size_t)TL));
  }
  const int ntile_all = (int)tiles.size();
  const size_t vec_bytes = (size_t)nn * 9 * TL * sizeof(T2);
  const int nvec = 8;   // U, UP, Y (rotating), T1, T3, Sa (S d x), TMP (d x), TV
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  int tpb = std::is_same<ST, double>::value ? 16 : 8;
  while (tpb > 1 && (size_t)tpb * nvec * vec_bytes > freeb / 2) tpb /= 2;
  if ((size_t)nvec * vec_bytes > freeb) { set_error("ed3: %d vectors of %zu bytes do not fit", nvec, vec_bytes); return ASR_ENOMEM; }
  tpb = std::min(tpb, ntile_all);
  const int npw = 4, npb = WPB * npw, bpt = (nn + npb - 1) / npb;
  const int nlp = tpb * TL;
  Dev<double> d_gblob, d_oc, d_na, d_nv, d_tn;
  Dev<GroupInfo> d_ginfo;
  ASR_TRY(d_gblob.alloc(gblob.size())); ASR_TRY(d_ginfo.alloc(ginfo.size())); ASR_TRY(d_oc.alloc(oc.size()));
  ASR_CUDA(cudaMemcpyAsync(d_gblob.p, gblob.data(), gblob.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_ginfo.p, ginfo.data(), ginfo.size() * sizeof(GroupInfo), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_oc.p, oc.data(), oc.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_TRY(d_na.alloc(nlp)); ASR_TRY(d_nv.alloc(nlp)); ASR_TRY(d_tn.alloc(nlp));
  Dev<int> d_lgroup, d_act, d_wact, d_m, d_tact, d_nfall, d_tgroup, d_kind, d_closed, d_lmap;
  Dev<double2> d_a, d_b, d_c, d_gprev, d_fprev, d_acur, d_bprev, d_su, d_sup, d_part, d_part2, d_z, d_g, d_f, d_sv, d_sa;
  ASR_TRY(d_lgroup.alloc(nlp)); ASR_TRY(d_act.alloc(nlp)); ASR_TRY(d_wact.alloc(nlp)); ASR_TRY(d_m.alloc(nlp));
  ASR_TRY(d_tact.alloc(tpb)); ASR_TRY(d_nfall.alloc(1)); ASR_TRY(d_tgroup.alloc(tpb)); ASR_TRY(d_kind.alloc(nlp));
  ASR_TRY(d_closed.alloc(nlp)); ASR_TRY(d_lmap.alloc(nlp));
  ASR_TRY(d_a.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_b.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_c.alloc((size_t)nlp * NLMAX));
  ASR_TRY(d_gprev.alloc(nlp)); ASR_TRY(d_fprev.alloc(nlp)); ASR_TRY(d_acur.alloc(nlp)); ASR_TRY(d_bprev.alloc(nlp));
  ASR_TRY(d_su.alloc(nlp)); ASR_TRY(d_sup.alloc(nlp)); ASR_TRY(d_z.alloc(nlp)); ASR_TRY(d_g.alloc(nlane)); ASR_TRY(d_f.alloc(nlane));
  ASR_TRY(d_part.alloc((size_t)tpb * bpt * TL)); ASR_TRY(d_part2.alloc((size_t)tpb * bpt * TL));
  ASR_TRY(d_sv.alloc(nlp)); ASR_TRY(d_sa.alloc(nlp));
  const size_t vlen = (size_t)tpb * nn * 9 * TL;
  std::vector<Dev<T2>> V(nvec);
  for (int q = 0; q < nvec; ++q) ASR_TRY(V[q].alloc(vlen));
  T2 *T1 = V[3].p, *T3 = V[4].p, *SA = V[5].p, *TMP = V[6].p, *TV = V[7].p;
  OpView ov = op->view();
  const ST* blk = std::is_same<ST, double>::value ? (const ST*)op->d_blocks : (const ST*)op->d_blocks_f;
  const size_t sm = smul_smem(op, sizeof(ST));
  g_out.assign(nlane, make_double2(0, 0));
  f_out.assign(nlane, make_double2(0, 0));
  na_out.assign(nlane, 0.0);
  nv_out.assign(nlane, 0.0);
  m_out.assign(nlane, 0);
  if (a_out) a_out->assign((size_t)nlane * NLMAX, make_double2(0, 0));
  if (b_out) b_out->assign((size_t)nlane * NLMAX, make_double2(0, 0));
  if (c_out) c_out->assign((size_t)nlane * NLMAX, make_double2(0, 0));
  std::vector<int> hgroup(nlp), lmap(nlp), hkind(nlp), hm(nlp);
  std::vector<double2> hz(nlp), hab((size_t)nlp * NLMAX);
  std::vector<double> hna(nlp), hnv(nlp);
  std::vector<double2> ones(nlp, make_double2(1.0, 0.0));
  ASR_CUDA(cudaMemsetAsync(d_nfall.p, 0, sizeof(int), s));
  // apply h' = g + d S d to x (raw): Sa = S d x (TMP for a species-dependent d), out = R_g x + d o Sa
  auto apply_hp = [&](const BatchView& bv, int grid, T2* x, T2* out) -> int {
    apply_SD<ST>(op, bv, dunif, x, TMP, SA, d_part.p, npw, grid, s);
    k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, SA, x, E3_G, false, x, false, nullptr, 1.0, false, out, d_part.p, npw);
    return ASR_OK;
  };
  for (int t0 = 0; t0 < ntile_all; t0 += tpb) {
    NvtxRange batch_range("ed3 batch");
    const int nt = std::min(tpb, ntile_all - t0);
    std::vector<int> tact(tpb, 0), act(nlp, 0), tgroup(tpb, -1);
    for (int q = 0; q < nlp; ++q) {
      int bt = q / TL, L = -1;
      if (bt < nt && q % TL < (int)tiles[t0 + bt].size()) L = tiles[t0 + bt][q % TL];
      lmap[q] = L;
      hgroup[q] = L >= 0 ? lane_group[L] : -1;
      hkind[q] = L >= 0 ? lane_kind[L] : 0;
      hz[q] = L >= 0 ? lane_z[L] : make_double2(0, 0);
      if (L >= 0) { tact[bt] = 1; act[q] = 1; tgroup[bt] = hgroup[q]; }
    }
    ASR_CUDA(cudaMemcpyAsync(d_lgroup.p, hgroup.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tgroup.p, tgroup.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_kind.p, hkind.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_lmap.p, lmap.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_act.p, act.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tact.p, tact.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_z.p, hz.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_su.p, ones.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemsetAsync(d_wact.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_m.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_closed.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_a.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_b.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_c.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_gprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_fprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_bprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_sup.p, 0, nlp * sizeof(double2), s));
    BatchView bv{nt, nn, op->nsmax, 0, ASR_MODE_EDC, project, tail, NLMAX, depth_tol, d_gblob.p, GL, d_ginfo.p, d_lgroup.p,
                 d_tgroup.p, d_z.p, d_act.p, d_wact.p, d_m.p, d_a.p, d_b.p, d_gprev.p, d_acur.p, d_bprev.p, d_su.p, d_sup.p,
                 d_tact.p, d_nfall.p, d_closed.p};
    const int grid = nt * bpt;
    const unsigned egrid = (unsigned)std::min<size_t>(65535, ((size_t)nt * nn * 9 * TL + 255) / 256);
    int kmax = 0;
    for (int q = 0; q < nlp; ++q) if (hgroup[q] >= 0) kmax = std::max(kmax, ginfo[hgroup[q]].nlev);
    // ---- start vectors (ed3_start, src/asr_ed3.f90:135-144): |v> = h'|e> (projected), |a> = |e> + o_c |v>
    k_init<ST><<<egrid, 256, 0, s>>>(bv, V[1].p, V[0].p);
    ASR_TRY(apply_hp(bv, grid, V[1].p, T1));
    if (project) k_project<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, T1, npw);
    k_ed3_dots<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, T1, d_oc.p, d_part.p, d_part2.p, npw);
    k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part.p, d_sv.p);
    k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part2.p, d_sa.p);
    std::vector<double2> hsv(nlp), hsa(nlp);
    ASR_CUDA(cudaMemcpyAsync(hsv.data(), d_sv.p, nlp * sizeof(double2), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaMemcpyAsync(hsa.data(), d_sa.p, nlp * sizeof(double2), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    std::vector<double> htn(nlp, 0.0);
    for (int q = 0; q < nlp; ++q) {
      hna[q] = hnv[q] = 1.0;
      if (hgroup[q] < 0) continue;
      double nv = std::sqrt(hsv[q].x), na = std::sqrt(hsa[q].x);   // sqrt(real(v.v)), as the reference
      if (!(nv >= 1.0e-14) || !(na >= 1.0e-14)) { set_error("ed3_start: zero start vector (group %d)", hgroup[q] + 1); return ASR_EINVAL; }
      hna[q] = na;
      hnv[q] = nv;
      htn[q] = hkind[q] == 0 ? nv : na;
    }
    ASR_CUDA(cudaMemcpyAsync(d_na.p, hna.data(), nlp * sizeof(double), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_nv.p, hnv.data(), nlp * sizeof(double), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tn.p, htn.data(), nlp * sizeof(double), cudaMemcpyHostToDevice, s));
    // V[0] = U_1 (scale 1), V[2] = U_0 = 0; T1 holds |v> until the start vectors are written
    k_ed3_start<ST><<<egrid, 256, 0, s>>>(bv, T1, d_oc.p, d_kind.p, d_na.p, d_nv.p, V[1].p, V[0].p, TV);
    // ---- the chains (chain, src/asr_ed3.f90:147-218)
    for (int k = 1; k <= kmax; ++k) {
      T2* U = V[k % 3].p;
      T2* UP = V[(k + 2) % 3].p;
      T2* Y = V[(k + 1) % 3].p;
      ASR_TRY(apply_hp(bv, grid, U, T1));                                              // t1 = h'u
      k_ed3_t3<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, U, T1, T3, npw);                  // t3 = u u - Qt t1
      apply_SD<ST>(op, bv, dunif, T3, TMP, SA, d_part.p, npw, grid, s);               // S d t3
      k_ed3_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, U, T1, T3, SA, TV, Y, d_part.p, d_part2.p, npw);
      k_ed3_reduce_a<<<nt, RED_THREADS, 0, s>>>(bv, d_part.p, d_part2.p, bpt, k, d_c.p, d_fprev.p, d_tn.p);
      k_lanczos_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, Y, U, UP, d_part.p, npw);
      k_reduce_b<<<nt, RED_THREADS, 0, s>>>(bv, d_part.p, bpt, k, 1.0e-12);
    }
    ASR_CUDA(cudaGetLastError());
    ctx->launches += 8 + (int64_t)kmax * (dunif ? 8 : 10);
    k_ed3_final<<<(nlp + 127) / 128, 128, 0, s>>>(bv, nlp, d_lmap.p, d_c.p, d_closed.p, d_g.p, d_f.p);
    ASR_CUDA(cudaMemcpyAsync(hm.data(), d_m.p, nlp * sizeof(int), cudaMemcpyDeviceToHost, s));
    for (int which = 0; which < 3; ++which) {
      std::vector<double2>* dst = which == 0 ? a_out : which == 1 ? b_out : c_out;
      if (!dst) continue;
      const double2* src = which == 0 ? d_a.p : which == 1 ? d_b.p : d_c.p;
      ASR_CUDA(cudaMemcpyAsync(hab.data(), src, hab.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
      ASR_CUDA(cudaStreamSynchronize(s));
      for (int q = 0; q < nlp; ++q)
        if (lmap[q] >= 0)
          std::copy(hab.begin() + (size_t)q * NLMAX, hab.begin() + (size_t)(q + 1) * NLMAX, dst->begin() + (size_t)lmap[q] * NLMAX);
    }
    ASR_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nlp; ++q) {
      int L = lmap[q];
      if (L < 0) continue;
      m_out[L] = hm[q];
      na_out[L] = hna[q];
      nv_out[L] = hnv[q];
    }
  }
  ASR_CUDA(cudaMemcpyAsync(g_out.data(), d_g.p, nlane * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(f_out.data(), d_f.p, nlane * sizeof(double2), cudaMemcpyDeviceToHost, s));
  int nf = 0;
  ASR_CUDA(cudaMemcpyAsync(&nf, d_nfall.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  ASR_CUDA(cudaGetLastError());
  ASR_TRY(check_wait_error(ctx));
  if (nfall_out) *nfall_out = nf;
  return ASR_OK;
}

// ================================================================================================ EPI block chains
// epi_blocks (src/asr_epi.f90:639-663): per symmetry-adapted start vector s0 (9 values on the start node, characters of
// the group in the lane group's chimask) two complex-symmetric chains on z - H(z) of the edc route, full depth: kind 0
// from s0 with the projection on |v> = h'|s0> (projected), kind 1 from |v> / |v| with the projection on s0; a chain that
// closes (|b| < 1e-12) gets no tail.  Per lane g and f = sum_k c_k pv_k, c_k = tv . u_k.

// U = s0 (node 0, 9 values of the lane's group), UP = 0
template <typename ST>
__global__ void k_epi_init(BatchView bv, const double* v9, typename St2<ST>::T* u, typename St2<ST>::T* up) {
  size_t n = (size_t)bv.ntile * bv.nn * 9 * TL;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int lane = (int)(q % TL);
    size_t rest = q / TL;
    int l = (int)(rest % 9);
    size_t nt = rest / 9;
    int node = (int)(nt % bv.nn);
    int tile = (int)(nt / bv.nn);
    int grp = bv.lane_group[tile * TL + lane];
    double v = (grp >= 0 && node == 0) ? v9[9 * grp + l] : 0.0;
    stv(u + q, make_double2(v, 0.0));
    stv(up + q, make_double2(0.0, 0.0));
  }
}

// kind 0: U = s0, TV = v; kind 1: U = v / nv, TV = s0 (s0 read from S0, v from VV), UP = 0
template <typename ST>
__global__ void k_epi_start(BatchView bv, const typename St2<ST>::T* __restrict__ S0, const typename St2<ST>::T* __restrict__ VV,
                            const int* kind, const double* nv, typename St2<ST>::T* U, typename St2<ST>::T* UP,
                            typename St2<ST>::T* TV) {
  size_t n = (size_t)bv.ntile * bv.nn * 9 * TL;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int lane = (int)(q % TL);
    int tile = (int)(q / ((size_t)bv.nn * 9 * TL));
    int L = tile * TL + lane;
    double2 u = make_double2(0, 0), t = make_double2(0, 0);
    if (bv.lane_group[L] >= 0) {
      double2 s0 = ld(S0 + q), v = ld(VV + q);
      if (kind[L] == 0) { u = s0; t = v; }
      else { u = cscale(v, 1.0 / nv[L]); t = s0; }
    }
    stv(U + q, u);
    stv(UP + q, make_double2(0, 0));
    stv(TV + q, t);
  }
}

// c_k = su * sum of the partial dots tv . X_k of this step
__global__ void k_epi_store_c(BatchView bv, const double2* part, int bpt, int k, double2* ccoef) {
  int tile = blockIdx.x, lane = threadIdx.x;
  if (tile >= bv.ntile || !bv.tile_act[tile]) return;
  const double2 c = block_sum_rows(part + (size_t)tile * bpt * TL, bpt, TL);
  if (lane >= TL) return;
  int L = tile * TL + lane;
  if (bv.lane_group[L] < 0 || !bv.lane_act[L]) return;
  ccoef[(size_t)L * NLMAX + k - 1] = cmul(c, bv.su[L]);
}

template <typename ST>
int run_epi_t(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
              const GroupLayout& GL, const std::vector<double>& v9, const std::vector<int>& lane_group,
              const std::vector<int>& lane_kind, const std::vector<double2>& lane_z, int tail, int project,
              std::vector<double2>& g_out, std::vector<double2>& f_out, std::vector<double>& nv_out, std::vector<int>& m_out,
              int64_t* nfall_out) {
  typedef typename St2<ST>::T T2;
  cudaStream_t s = ctx->stream;
  const int nn = op->nn, nlane = (int)lane_group.size();
  bool dunif = true, any_o = false;
  for (auto& g : ginfo) {
    if (!(g.flags & GF_D_UNIFORM)) dunif = false;
    if (!(g.flags & GF_O_ZERO)) any_o = true;
    if (g.nlev > NLMAX) { set_error("epi_blocks: depth %d above %d", g.nlev, NLMAX); return ASR_EINVAL; }
  }
  const bool fused = dunif && !any_o;
  std::vector<std::vector<int>> tiles;
  {
    std::vector<std::vector<int>> per_group(ginfo.size());
    for (int L = 0; L < nlane; ++L) per_group[lane_group[L]].push_back(L);
    for (auto& lst : per_group)
      for (size_t q = 0; q < lst.size(); q += TL)
        tiles.emplace_back(lst.begin() + q, lst.begin() + std::min(lst.size(), q + (size_t)TL));
  }
  const int ntile_all = (int)tiles.size();
  const size_t vec_bytes = (size_t)nn * 9 * TL * sizeof(T2);
  const int nvec = 3 + 1 + 4 + 2;   // U, UP, Y (rotating), TV, four step temporaries, S d x and d x of h'
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  int tpb = std::is_same<ST, double>::value ? 16 : 8;
  while (tpb > 1 && (size_t)tpb * nvec * vec_bytes > freeb / 2) tpb /= 2;
  if ((size_t)nvec * vec_bytes > freeb) { set_error("epi_blocks: %d vectors of %zu bytes do not fit", nvec, vec_bytes); return ASR_ENOMEM; }
  tpb = std::min(tpb, ntile_all);
  const int npw = 4, npb = WPB * npw, bpt = (nn + npb - 1) / npb;
  const int nlp = tpb * TL;
  Dev<double> d_gblob, d_v9, d_nv;
  Dev<GroupInfo> d_ginfo;
  ASR_TRY(d_gblob.alloc(gblob.size())); ASR_TRY(d_ginfo.alloc(ginfo.size())); ASR_TRY(d_v9.alloc(v9.size()));
  ASR_CUDA(cudaMemcpyAsync(d_gblob.p, gblob.data(), gblob.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_ginfo.p, ginfo.data(), ginfo.size() * sizeof(GroupInfo), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_v9.p, v9.data(), v9.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_TRY(d_nv.alloc(nlp));
  Dev<int> d_lgroup, d_act, d_wact, d_m, d_tact, d_nfall, d_tgroup, d_kind, d_closed, d_lmap;
  Dev<double2> d_a, d_b, d_c, d_gprev, d_acur, d_bprev, d_su, d_sup, d_part, d_part2, d_z, d_g, d_f, d_sv;
  ASR_TRY(d_lgroup.alloc(nlp)); ASR_TRY(d_act.alloc(nlp)); ASR_TRY(d_wact.alloc(nlp)); ASR_TRY(d_m.alloc(nlp));
  ASR_TRY(d_tact.alloc(tpb)); ASR_TRY(d_nfall.alloc(1)); ASR_TRY(d_tgroup.alloc(tpb)); ASR_TRY(d_kind.alloc(nlp));
  ASR_TRY(d_closed.alloc(nlp)); ASR_TRY(d_lmap.alloc(nlp));
  ASR_TRY(d_a.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_b.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_c.alloc((size_t)nlp * NLMAX));
  ASR_TRY(d_gprev.alloc(nlp)); ASR_TRY(d_acur.alloc(nlp)); ASR_TRY(d_bprev.alloc(nlp)); ASR_TRY(d_su.alloc(nlp));
  ASR_TRY(d_sup.alloc(nlp)); ASR_TRY(d_z.alloc(nlp)); ASR_TRY(d_g.alloc(nlane)); ASR_TRY(d_f.alloc(nlane));
  ASR_TRY(d_part.alloc((size_t)tpb * bpt * TL)); ASR_TRY(d_part2.alloc((size_t)tpb * bpt * TL)); ASR_TRY(d_sv.alloc(nlp));
  const size_t vlen = (size_t)tpb * nn * 9 * TL;
  std::vector<Dev<T2>> V(nvec);
  for (int q = 0; q < nvec; ++q) ASR_TRY(V[q].alloc(vlen));
  T2 *TV = V[3].p, *W1 = V[4].p, *W2 = V[5].p, *W3 = V[6].p, *W4 = V[7].p, *SA = V[8].p, *TMP = V[9].p;
  OpView ov = op->view();
  g_out.assign(nlane, make_double2(0, 0));
  f_out.assign(nlane, make_double2(0, 0));
  nv_out.assign(nlane, 0.0);
  m_out.assign(nlane, 0);
  std::vector<int> hgroup(nlp), lmap(nlp), hkind(nlp), hm(nlp);
  std::vector<double2> hz(nlp), ones(nlp, make_double2(1.0, 0.0));
  std::vector<double> hnv(nlp);
  ASR_CUDA(cudaMemsetAsync(d_nfall.p, 0, sizeof(int), s));
  for (int t0 = 0; t0 < ntile_all; t0 += tpb) {
    NvtxRange batch_range("epi batch");
    const int nt = std::min(tpb, ntile_all - t0);
    std::vector<int> tact(tpb, 0), act(nlp, 0), tgroup(tpb, -1);
    for (int q = 0; q < nlp; ++q) {
      int bt = q / TL, L = -1;
      if (bt < nt && q % TL < (int)tiles[t0 + bt].size()) L = tiles[t0 + bt][q % TL];
      lmap[q] = L;
      hgroup[q] = L >= 0 ? lane_group[L] : -1;
      hkind[q] = L >= 0 ? lane_kind[L] : 0;
      hz[q] = L >= 0 ? lane_z[L] : make_double2(0, 0);
      if (L >= 0) { tact[bt] = 1; act[q] = 1; tgroup[bt] = hgroup[q]; }
    }
    ASR_CUDA(cudaMemcpyAsync(d_lgroup.p, hgroup.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tgroup.p, tgroup.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_kind.p, hkind.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_lmap.p, lmap.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_act.p, act.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tact.p, tact.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_z.p, hz.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_su.p, ones.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemsetAsync(d_wact.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_m.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_closed.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_a.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_b.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_c.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_gprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_bprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_sup.p, 0, nlp * sizeof(double2), s));
    BatchView bv{nt, nn, op->nsmax, 0, ASR_MODE_EDC, project, tail, NLMAX, 0.0, d_gblob.p, GL, d_ginfo.p, d_lgroup.p,
                 d_tgroup.p, d_z.p, d_act.p, d_wact.p, d_m.p, d_a.p, d_b.p, d_gprev.p, d_acur.p, d_bprev.p, d_su.p, d_sup.p,
                 d_tact.p, d_nfall.p, d_closed.p};
    const int grid = nt * bpt;
    const unsigned egrid = (unsigned)std::min<size_t>(65535, ((size_t)nt * nn * 9 * TL + 255) / 256);
    int kmax = 0;
    for (int q = 0; q < nlp; ++q) if (hgroup[q] >= 0) kmax = std::max(kmax, ginfo[hgroup[q]].nlev);
    // ---- start vectors (epi_start, src/asr_epi.f90:578-587): s0 on the start node, |v> = h'|s0> projected, |v|
    k_epi_init<ST><<<egrid, 256, 0, s>>>(bv, d_v9.p, W1, V[0].p);
    apply_SD<ST>(op, bv, dunif, W1, TMP, SA, d_part.p, npw, grid, s);
    k_combine<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, SA, W1, E3_G, false, W1, false, nullptr, 1.0, false, W2, d_part.p, npw);
    if (project) k_project<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, W2, npw);
    k_dot<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, W2, W2, d_part.p, npw);
    k_lane_sum<<<nt, RED_THREADS, 0, s>>>(nt, bpt, d_tact.p, d_part.p, d_sv.p);
    std::vector<double2> hsv(nlp);
    ASR_CUDA(cudaMemcpyAsync(hsv.data(), d_sv.p, nlp * sizeof(double2), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nlp; ++q) {
      hnv[q] = 1.0;
      if (hgroup[q] < 0) continue;
      double nv = std::sqrt(hsv[q].x);   // sqrt(real(v . v)), as the reference
      if (!(nv >= 1.0e-14)) { set_error("epi_start: zero start vector (group %d)", hgroup[q] + 1); return ASR_EINVAL; }
      hnv[q] = nv;
    }
    ASR_CUDA(cudaMemcpyAsync(d_nv.p, hnv.data(), nlp * sizeof(double), cudaMemcpyHostToDevice, s));
    k_epi_start<ST><<<egrid, 256, 0, s>>>(bv, W1, W2, d_kind.p, d_nv.p, V[1].p, V[0].p, TV);
    // ---- the chains (chain, src/asr_epi.f90:588-636): full depth, projections c_k = tv . u_k
    for (int k = 1; k <= kmax; ++k) {
      bv.kstep = k;
      T2* U = V[k % 3].p;
      T2* UP = V[(k + 2) % 3].p;
      T2* Y = V[(k + 1) % 3].p;
      k_dot<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, TV, U, d_part2.p, npw);
      k_epi_store_c<<<nt, RED_THREADS, 0, s>>>(bv, d_part2.p, bpt, k, d_c.p);
      ASR_TRY(step_apply<ST>(ctx, op, bv, fused, any_o, dunif, U, Y, W1, W2, W3, W4, d_part.p, npw, grid));
      k_reduce_a<<<nt, RED_THREADS, 0, s>>>(bv, d_part.p, bpt, k);
      k_lanczos_w<ST><<<grid, WPB * TL, 0, s>>>(ov, bv, Y, U, UP, d_part.p, npw);
      k_reduce_b<<<nt, RED_THREADS, 0, s>>>(bv, d_part.p, bpt, k, 1.0e-12);
    }
    ASR_CUDA(cudaGetLastError());
    ctx->launches += 8 + (int64_t)kmax * (5 + (fused ? 1 : (any_o ? 7 : (dunif ? 2 : 3))));
    k_ed3_final<<<(nlp + 127) / 128, 128, 0, s>>>(bv, nlp, d_lmap.p, d_c.p, d_closed.p, d_g.p, d_f.p);
    ASR_CUDA(cudaMemcpyAsync(hm.data(), d_m.p, nlp * sizeof(int), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nlp; ++q) {
      int L = lmap[q];
      if (L < 0) continue;
      m_out[L] = hm[q];
      nv_out[L] = hnv[q];
    }
  }
  ASR_CUDA(cudaMemcpyAsync(g_out.data(), d_g.p, nlane * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(f_out.data(), d_f.p, nlane * sizeof(double2), cudaMemcpyDeviceToHost, s));
  int nf = 0;
  ASR_CUDA(cudaMemcpyAsync(&nf, d_nfall.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  ASR_CUDA(cudaGetLastError());
  ASR_TRY(check_wait_error(ctx));
  if (nfall_out) *nfall_out = nf;
  return ASR_OK;
}

}  // namespace

// the operator kernels stage up to 96 KB of bond blocks in shared memory (set once per device)
static void smem_attrs() {
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaFuncSetAttribute(k_smul<double, true, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, true, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, false, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, false, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, true, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, true, true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, true, true, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, true, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, true, true, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<double, true, true, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, true, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul<float, true, true, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
  cudaFuncSetAttribute(k_smul_bulk<double, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_smul_bulk<double, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_smul_bulk<double, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_smul_bulk<float, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_smul_bulk<float, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_smul_bulk<float, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  done[dev] = true;
}

int run_adjoint(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                const GroupLayout& GL, const std::vector<int>& lane_group, const std::vector<double2>& lane_z,
                const std::vector<double2>& lane_w, double depth_tol, int tail, int project, int stride, int precision,
                std::vector<double2>& g_out, std::vector<int>& m_out, std::vector<double2>& grad_out) {
  smem_attrs();
  if (smul_smem(op, sizeof(double)) > 96 * 1024) { set_error("adjoint: bond tables above 96 KB of shared memory"); return ASR_EINVAL; }
  if (precision == ASR_FP32)
    return run_adjoint_t<float>(ctx, op, ginfo, gblob, GL, lane_group, lane_z, lane_w, depth_tol, tail, project, stride, g_out,
                                m_out, grad_out);
  return run_adjoint_t<double>(ctx, op, ginfo, gblob, GL, lane_group, lane_z, lane_w, depth_tol, tail, project, stride, g_out,
                               m_out, grad_out);
}

int run_ed3(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
            const GroupLayout& GL, const std::vector<double>& oc, const std::vector<int>& lane_group,
            const std::vector<int>& lane_kind, const std::vector<double2>& lane_z, double depth_tol, int tail, int project,
            int precision, std::vector<double2>& g_out, std::vector<double2>& f_out, std::vector<double>& na_out,
            std::vector<double>& nv_out, std::vector<int>& m_out, std::vector<double2>* a_out, std::vector<double2>* b_out,
            std::vector<double2>* c_out, int64_t* nfall_out) {
  smem_attrs();
  if (smul_smem(op, sizeof(double)) > 96 * 1024) { set_error("ed3: bond tables above 96 KB of shared memory"); return ASR_EINVAL; }
  if (precision == ASR_FP32)
    return run_ed3_t<float>(ctx, op, ginfo, gblob, GL, oc, lane_group, lane_kind, lane_z, depth_tol, tail, project, g_out, f_out,
                            na_out, nv_out, m_out, a_out, b_out, c_out, nfall_out);
  return run_ed3_t<double>(ctx, op, ginfo, gblob, GL, oc, lane_group, lane_kind, lane_z, depth_tol, tail, project, g_out, f_out,
                           na_out, nv_out, m_out, a_out, b_out, c_out, nfall_out);
}

int run_epi(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
            const GroupLayout& GL, const std::vector<double>& v9, const std::vector<int>& lane_group,
            const std::vector<int>& lane_kind, const std::vector<double2>& lane_z, int tail, int project, int precision,
            std::vector<double2>& g_out, std::vector<double2>& f_out, std::vector<double>& nv_out, std::vector<int>& m_out,
            int64_t* nfall_out) {
  smem_attrs();
  if (smul_smem(op, sizeof(double)) > 96 * 1024) { set_error("epi_blocks: bond tables above 96 KB of shared memory"); return ASR_EINVAL; }
  if (precision == ASR_FP32)
    return run_epi_t<float>(ctx, op, ginfo, gblob, GL, v9, lane_group, lane_kind, lane_z, tail, project, g_out, f_out, nv_out,
                            m_out, nfall_out);
  return run_epi_t<double>(ctx, op, ginfo, gblob, GL, v9, lane_group, lane_kind, lane_z, tail, project, g_out, f_out, nv_out,
                           m_out, nfall_out);
}

int run_lanes(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
              const GroupLayout& GL, const std::vector<int>& lane_group, const double2* d_lane_z, int nlane,
              const RunOptions& opt, double2* d_g_out, std::vector<double2>* a_out, std::vector<double2>* b_out,
              std::vector<int>* m_out, int64_t* nfall_out, int64_t* nsteps_out, const ProjSpec* proj, double* dev_ms) {
  smem_attrs();
  if (smul_smem(op, sizeof(double)) > 96 * 1024) { set_error("chains: bond tables above 96 KB of shared memory"); return ASR_EINVAL; }
  if (opt.precision == ASR_FP32)
    return run_lanes_t<float>(ctx, op, ginfo, gblob, GL, lane_group, d_lane_z, nlane, opt, d_g_out, a_out, b_out, m_out, nfall_out,
                              nsteps_out, proj, dev_ms);
  return run_lanes_t<double>(ctx, op, ginfo, gblob, GL, lane_group, d_lane_z, nlane, opt, d_g_out, a_out, b_out, m_out, nfall_out,
                             nsteps_out, proj, dev_ms);
}

// ------------------------------------------------------------------------------------------------ drop-in applications
int apply_vectors(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                  const GroupLayout& GL, int nvec, const double* x_host, bool complex_in, double* y_host, int what) {
  smem_attrs();
  cudaStream_t s = ctx->stream;
  const int nn = op->nn;
  const int nt = (nvec + TL - 1) / TL;
  const size_t nel = (size_t)nt * nn * 9 * TL;
  // normalised coordinates in and out; the kernels work in amplitude coordinates (x / sqrt(orbit size))
  std::vector<double> sqv(nn);
  ASR_CUDA(cudaMemcpyAsync(sqv.data(), op->d_sq, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  std::vector<double2> hx(nel, make_double2(0, 0));
  for (int v = 0; v < nvec; ++v)
    for (int i = 0; i < nn; ++i)
      for (int l = 0; l < 9; ++l) {   // user vectors in the reference numbering, device rows in the device node order
        const int n = op->dev_node(i);
        size_t src = (size_t)v * 9 * nn + 9 * (size_t)i + l;
        size_t dst = (((size_t)(v / TL) * nn + n) * 9 + l) * TL + v % TL;
        double f = what == APPLY_PROJECT ? 1.0 : 1.0 / sqv[n];
        hx[dst] = complex_in ? make_double2(f * x_host[2 * src], f * x_host[2 * src + 1]) : make_double2(f * x_host[src], 0.0);
      }
  Dev<double> d_gblob;
  Dev<GroupInfo> d_ginfo;
  ASR_TRY(d_gblob.alloc(gblob.size()));
  ASR_TRY(d_ginfo.alloc(ginfo.size()));
  ASR_CUDA(cudaMemcpyAsync(d_gblob.p, gblob.data(), gblob.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_ginfo.p, ginfo.data(), ginfo.size() * sizeof(GroupInfo), cudaMemcpyHostToDevice, s));
  const int nlp = nt * TL;
  const int npw = 4, npb = WPB * npw, bpt = (nn + npb - 1) / npb;
  std::vector<int> hgroup(nlp), ones(nlp, 1), tact(nt, 1), tgroup(nt, 0);
  for (int q = 0; q < nlp; ++q) hgroup[q] = q < nvec ? 0 : -1;
  std::vector<double2> hz(nlp, make_double2(0.0, what == APPLY_RAND_Z ? 1.0 : 0.0)), hsu(nlp, make_double2(1.0, 0.0));
  Dev<int> d_lgroup, d_act, d_tact, d_tgroup;
  Dev<double2> d_z, d_su, d_part, V[6];
  ASR_TRY(d_lgroup.alloc(nlp)); ASR_TRY(d_act.alloc(nlp)); ASR_TRY(d_tact.alloc(nt)); ASR_TRY(d_z.alloc(nlp));
  ASR_TRY(d_tgroup.alloc(nt));
  ASR_CUDA(cudaMemcpyAsync(d_tgroup.p, tgroup.data(), nt * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_TRY(d_su.alloc(nlp)); ASR_TRY(d_part.alloc((size_t)nt * bpt * TL));
  for (int q = 0; q < 6; ++q) ASR_TRY(V[q].alloc(nel));
  ASR_CUDA(cudaMemcpyAsync(V[0].p, hx.data(), nel * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_lgroup.p, hgroup.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_act.p, ones.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_tact.p, tact.data(), nt * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_z.p, hz.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_su.p, hsu.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
  BatchView bv{};
  bv.ntile = nt; bv.nn = nn; bv.nsm = op->nsmax; bv.mode = ASR_MODE_EDC; bv.project = 1; bv.gblob = d_gblob.p; bv.GL = GL;
  bv.ginfo = d_ginfo.p; bv.lane_group = d_lgroup.p; bv.tile_group = d_tgroup.p; bv.lane_z = d_z.p; bv.lane_act = d_act.p; bv.lane_wact = d_act.p;
  bv.su = d_su.p; bv.sup = d_su.p; bv.tile_act = d_tact.p;
  const int grid = nt * bpt;
  OpView ov = op->view();
  double2* OUT = V[1].p;
  if (what == APPLY_H) {
    bool any_o = !(ginfo[0].flags & GF_O_ZERO), dunif = ginfo[0].flags & GF_D_UNIFORM;
    bool fused = dunif && !any_o;
    ASR_TRY(step_apply<double>(ctx, op, bv, fused, any_o, dunif, V[0].p, V[1].p, V[2].p, V[3].p, V[4].p, V[5].p, d_part.p, npw,
                               grid));
  } else if (what == APPLY_RAND_Z) {
    // w = X x with X = z pa + pb, z = i: the complex parameter par = pb + i pa
    k_combine<double><<<grid, WPB * TL, 0, s>>>(ov, bv, nullptr, V[0].p, PB, true, V[0].p, false, nullptr, 1.0, true, V[1].p,
                                                d_part.p, npw);
  } else {
    k_project<double><<<grid, WPB * TL, 0, s>>>(ov, bv, V[0].p, npw);
    OUT = V[0].p;
  }
  ASR_CUDA(cudaGetLastError());
  std::vector<double2> hy(nel);
  ASR_CUDA(cudaMemcpyAsync(hy.data(), OUT, nel * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  ASR_CUDA(cudaGetLastError());
  for (int v = 0; v < nvec; ++v)
    for (int i = 0; i < nn; ++i)
      for (int l = 0; l < 9; ++l) {
        const int n = op->dev_node(i);
        size_t dst = (size_t)v * 9 * nn + 9 * (size_t)i + l;
        double2 val = hy[(((size_t)(v / TL) * nn + n) * 9 + l) * TL + v % TL];
        if (what != APPLY_PROJECT) val = cscale(val, sqv[n]);
        if (complex_in || what != APPLY_H) { y_host[2 * dst] = val.x; y_host[2 * dst + 1] = val.y; }
        else y_host[dst] = val.x;
      }
  return ASR_OK;
}

}  // namespace asrb
