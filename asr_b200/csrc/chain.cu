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
// node-parallel kernels; with d uniform and o = 0 (the edc route) it is one fused kernel: y = sq (d S d x0 +
// (c + e + X(z)) x0) with x0 = u / sq and the dot a = u . y.  Vectors are kept unnormalised with a complex scale per
// lane (u = s U); every kernel works on U and applies s once per node, which turns the normalisation u = w / b into a
// scalar update.  Reductions (a, b) are per block partial sums in a fixed order followed by a per-tile pass, so the
// result is bitwise the same in every run.
#include <algorithm>
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

__device__ __forceinline__ size_t vix(int tile, int nn, int node, int l) {
  return (((size_t)tile * nn + node) * 9 + l) * TL;
}

// complex weight of the diagonal term p (+ X(z) if withx) for (l, own, flip) of class kap
__device__ __forceinline__ double2 pweight(const double* gb, const GroupLayout& GL, int p, bool withx, double2 z, int nsm,
                                           int kap, int own, int flip, int l) {
  int q = ((kap * nsm + own) * nsm + flip) * 9 + l;
  double w = p >= 0 ? __ldg(gb + GL.w(p) + q) : 0.0;
  if (withx) {
    double wa = __ldg(gb + GL.w(PA) + q);
    return make_double2(w + z.x * wa, z.y * wa);
  }
  return make_double2(w, 0.0);
}
__device__ __forceinline__ double2 praw(const double* gb, const GroupLayout& GL, int p, bool withx, double2 z, int sp, int l) {
  int q = (sp - 1) * 9 + l;
  double w = p >= 0 ? __ldg(gb + GL.raw(p) + q) : 0.0;
  if (withx) {
    double wa = __ldg(gb + GL.raw(PA) + q);
    return make_double2(w + z.x * wa, z.y * wa);
  }
  return make_double2(w, 0.0);
}
__device__ __forceinline__ int frozen_of(const OpView& op, const GroupInfo& gi, int i) {
  return (op.start[i] && gi.frozen_sp > 0) ? gi.frozen_sp : (int)op.frozen[i];
}

// R_p(x) at node i for one lane: the random site-diagonal operator of apply_rand (src/asr_augcls.f90:380-403) on the
// vector v (unscaled); norm: v is in normalised coordinates (x = v / sq), else amplitude coordinates.
template <typename T2>
__device__ __forceinline__ void rand_term(const OpView& op, const GroupInfo& gi, const double* gb, const GroupLayout& GL, int p,
                                          bool withx, double2 z, const T2* v, int tile, int i, int lane, bool norm, double2* out,
                                          const double2* xi_own) {
  int fs = frozen_of(op, gi, i);
  if (fs > 0) {
    for (int l = 0; l < 9; ++l) out[l] = cmul(praw(gb, GL, p, withx, z, fs, l), xi_own[l]);
    return;
  }
  const int nsm = op.nsmax;
  int kap = op.ncl[i], l0 = op.lst[i];
  for (int l = 0; l < 9; ++l) out[l] = cmul(pweight(gb, GL, p, withx, z, nsm, kap, l0, l0, l), xi_own[l]);
  int nk = op.nsc[kap];
  for (int k = 0; k < nk; ++k) {
    if (k == l0) continue;
    int r = op.flipr[k + nsm * i];
    if (r < 0) continue;
    int g = op.flipg[k + nsm * i];
    double f = norm ? op.isq[r] : 1.0;
    bool neg = (gi.chimask >> g) & 1ull;
    uint32_t sgm = op.sgm[g];
    for (int l = 0; l < 9; ++l) {
      int pl = op.pi[g * 9 + l];
      double2 x = ld(v + vix(tile, op.nn, r, pl) + lane);
      double sgn = (((sgm >> l) & 1u) ^ (neg ? 1u : 0u)) ? -f : f;
      out[l] = cadd(out[l], cmul(pweight(gb, GL, p, withx, z, nsm, kap, l0, k, l), cscale(x, sgn)));
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

// ------------------------------------------------------------------------------------------------ S application
// t2 = S t1 (src/asr_augcls.f90:456-477 / src/asr_augblk.f90:170-203), unscaled amplitude coordinates.
// FUSE_D: t1 = d o (U / sq) is formed on the fly from the current vector U (d uniform per orbital).
// FINAL (needs FUSE_D, o = 0): y = s sq (d o t2 + (c + e + X(z)) x0) and the partial dot U . y.
template <typename ST, bool FUSE_D, bool FINAL>
__global__ void __launch_bounds__(WPB * TL) k_smul(OpView op, BatchView bv, const ST* __restrict__ blocks,
                                                   const typename St2<ST>::T* __restrict__ in,
                                                   typename St2<ST>::T* __restrict__ out, double2* part, int npw) {
  typedef typename St2<ST>::T T2;
  extern __shared__ unsigned char smem_raw[];
  const int ns1 = op.nslot + 1;
  ST* Bs = (ST*)smem_raw;                                        // [ntype][ns1][81]
  uint8_t* pis = (uint8_t*)(Bs + (size_t)op.ntype * ns1 * 81);  // [nop][9]
  uint16_t* sgs = (uint16_t*)(pis + ((op.nop * 9 + 1) & ~1));    // [nop]
  double* dds = (double*)(((uintptr_t)(sgs + op.nop) + 15) & ~(uintptr_t)15);   // [TL][9]
  NodeIter it;
  int bpt;
  bool live = node_iter(bv, npw, it, bpt);
  for (int q = threadIdx.x; q < op.ntype * ns1 * 81; q += blockDim.x) Bs[q] = blocks[q];
  for (int q = threadIdx.x; q < op.nop * 9; q += blockDim.x) pis[q] = op.pi[q];
  for (int q = threadIdx.x; q < op.nop; q += blockDim.x) sgs[q] = op.sgm[q];
  const int lane = threadIdx.x % TL, w = threadIdx.x / TL;
  const int L = it.tile * TL + lane;
  const int grp = live ? bv.lane_group[L] : -1;
  unsigned long long chimask = 0ull;
  int gflags = 0, gfrozen = 0;
  if (grp >= 0) {
    chimask = bv.ginfo[grp].chimask;
    gflags = bv.ginfo[grp].flags;
    gfrozen = bv.ginfo[grp].frozen_sp;
  }
  if (w == 0)
    for (int l = 0; l < 9; ++l) dds[lane * 9 + l] = grp >= 0 ? bv.ginfo[grp].dd[l] : 0.0;
  __syncthreads();
  if (!live) return;
  double2 dot = make_double2(0.0, 0.0);
  for (int qn = 0; qn < npw; ++qn) {
    int i = it.first + w + WPB * qn;
    if (i >= bv.nn) break;
    const ST* B = Bs + (size_t)op.typ[i] * ns1 * 81;
    T2 acc[9];
    for (int l = 0; l < 9; ++l) { acc[l].x = 0; acc[l].y = 0; }
    {   // on-site block: own node, t1 = d o (U / sq) (FUSE_D) or t1
      const ST f = FUSE_D ? (ST)op.isq[i] : (ST)1;
      const T2* src = in + vix(it.tile, bv.nn, i, 0) + lane;
      T2 v[9];
      for (int l2 = 0; l2 < 9; ++l2) {
        T2 x = src[l2 * TL];
        ST fl = FUSE_D ? f * (ST)dds[lane * 9 + l2] : f;
        v[l2].x = x.x * fl;
        v[l2].y = x.y * fl;
      }
      for (int l2 = 0; l2 < 9; ++l2)
        for (int l = 0; l < 9; ++l) {
          ST bb = B[l * 9 + l2];
          acc[l].x = fma_(bb, v[l2].x, acc[l].x);
          acc[l].y = fma_(bb, v[l2].y, acc[l].y);
        }
    }
    for (int k = 0; k < op.nslot; ++k) {
      int r = op.hopr[k + op.nslot * i];
      if (r < 0) continue;
      int g = op.hopg[k + op.nslot * i];
      const uint32_t sgm = sgs[g];
      const bool neg = (chimask >> g) & 1ull;
      const ST f = FUSE_D ? (ST)op.isq[r] : (ST)1;
      const T2* src = in + vix(it.tile, bv.nn, r, 0) + lane;
      T2 v[9];
      for (int lp = 0; lp < 9; ++lp) {
        int p = pis[g * 9 + lp];
        T2 x = src[p * TL];
        ST fl = FUSE_D ? f * (ST)dds[lane * 9 + p] : f;
        if (((sgm >> lp) & 1u) ^ (neg ? 1u : 0u)) fl = -fl;
        v[lp].x = x.x * fl;
        v[lp].y = x.y * fl;
      }
      const ST* Bk = B + (size_t)(k + 1) * 81;
      for (int l = 0; l < 9; ++l)
        for (int lp = 0; lp < 9; ++lp) {
          ST bb = Bk[l * 9 + lp];
          acc[l].x = fma_(bb, v[lp].x, acc[l].x);
          acc[l].y = fma_(bb, v[lp].y, acc[l].y);
        }
    }
    if (!FINAL) {
      for (int l = 0; l < 9; ++l) stv(out + vix(it.tile, bv.nn, i, l) + lane, make_double2(acc[l].x, acc[l].y));
    } else {
      // y_l = s sq (d_l t2_l + P_l(x0)),  P = c + e + X(z) (src/asr_augblk.f90:219-250), orbital by orbital
      const double* gb = bv.gblob + (size_t)(grp >= 0 ? grp : 0) * bv.GL.stride;
      const double2 z = bv.lane_z[L];
      const double2 s = bv.su[L];
      const bool withx = !(gflags & GF_X_ZERO);
      const double sqi = op.sq[i], isqi = op.isq[i];
      const int fs = (op.start[i] && gfrozen > 0) ? gfrozen : (int)op.frozen[i];
      const int nsm = op.nsmax, kap = op.ncl[i], l0 = op.lst[i], nk = op.nsc[kap];
      for (int l = 0; l < 9; ++l) {
        double2 ui = ld(in + vix(it.tile, bv.nn, i, l) + lane);
        double2 x0 = cscale(ui, isqi);
        double2 pt;
        if (fs > 0) {
          pt = cmul(praw(gb, bv.GL, PCEB, withx, z, fs, l), x0);
        } else {
          pt = cmul(pweight(gb, bv.GL, PCEB, withx, z, nsm, kap, l0, l0, l), x0);
          for (int k = 0; k < nk; ++k) {
            if (k == l0) continue;
            int r = op.flipr[k + nsm * i];
            if (r < 0) continue;
            int g = op.flipg[k + nsm * i];
            bool neg = (chimask >> g) & 1ull;
            double fr = ((((uint32_t)sgs[g] >> l) & 1u) ^ (neg ? 1u : 0u)) ? -op.isq[r] : op.isq[r];
            double2 xr = cscale(ld(in + vix(it.tile, bv.nn, r, pis[g * 9 + l]) + lane), fr);
            pt = cadd(pt, cmul(pweight(gb, bv.GL, PCEB, withx, z, nsm, kap, l0, k, l), xr));
          }
        }
        double2 h = cscale(make_double2(acc[l].x, acc[l].y), dds[lane * 9 + l]);
        double2 y = cmul(s, cscale(cadd(h, pt), sqi));
        stv(out + vix(it.tile, bv.nn, i, l) + lane, y);
        dot = cadd(dot, cmul(cmul(s, ui), y));
      }
    }
  }
  if (FINAL) block_reduce_store(dot, part, it.tile, bpt);
}

// ------------------------------------------------------------------------------------------------ random operators
// out = R_p(in) (unscaled amplitude coordinates); norm: in is U (normalised coordinates)
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_rand(OpView op, BatchView bv, int p, const typename St2<ST>::T* __restrict__ in,
                                                   bool norm, typename St2<ST>::T* __restrict__ out, int npw) {
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
    double f = norm ? op.isq[i] : 1.0;
    for (int l = 0; l < 9; ++l) xi[l] = cscale(ld(in + vix(it.tile, bv.nn, i, l) + lane), f);
    rand_term(op, gi, gb, bv.GL, p, false, make_double2(0, 0), in, it.tile, i, lane, norm, o, xi);
    for (int l = 0; l < 9; ++l) stv(out + vix(it.tile, bv.nn, i, l) + lane, o[l]);
  }
}

// out = sgnAB (A + B) + C + H, A = D t2 (uniform: d o t2), B = R_pB(v1), C = R_(e+pb) + z pa on x0 (optional),
// H = h1 (optional).  final: y = s sq out, partial dot U . y; else out is written unscaled (amplitude coordinates).
template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_combine(OpView op, BatchView bv, const typename St2<ST>::T* __restrict__ t2,
                                                      const typename St2<ST>::T* __restrict__ v1, bool v1norm, int pB, bool bx,
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
          else rand_term(op, gi, gb, bv.GL, PD, false, z, t2, it.tile, i, lane, false, acc, xi);
        } else {
          for (int l = 0; l < 9; ++l) acc[l] = make_double2(0, 0);
        }
        if (v1) {
          double f = v1norm ? op.isq[i] : 1.0;
          for (int l = 0; l < 9; ++l) xi[l] = cscale(ld(v1 + vix(it.tile, bv.nn, i, l) + lane), f);
          rand_term(op, gi, gb, bv.GL, pB, bx, z, v1, it.tile, i, lane, v1norm, tmp, xi);
          for (int l = 0; l < 9; ++l) acc[l] = cadd(acc[l], tmp[l]);
        }
        for (int l = 0; l < 9; ++l) acc[l] = cscale(acc[l], sgnAB);
        double2 ui[9];
        for (int l = 0; l < 9; ++l) ui[l] = ld(u + vix(it.tile, bv.nn, i, l) + lane);
        if (cterm) {
          for (int l = 0; l < 9; ++l) xi[l] = cscale(ui[l], op.isq[i]);
          rand_term(op, gi, gb, bv.GL, PEB, !(gi.flags & GF_X_ZERO), z, u, it.tile, i, lane, true, tmp, xi);
          for (int l = 0; l < 9; ++l) acc[l] = cadd(acc[l], tmp[l]);
        }
        if (h1) for (int l = 0; l < 9; ++l) acc[l] = cadd(acc[l], ld(h1 + vix(it.tile, bv.nn, i, l) + lane));
        if (final_) {
          double sqi = op.sq[i];
          for (int l = 0; l < 9; ++l) {
            double2 y = cmul(s, cscale(acc[l], sqi));
            stv(out + vix(it.tile, bv.nn, i, l) + lane, y);
            dot = cadd(dot, cmul(cmul(s, ui[l]), y));
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
// src/asr_augcls.f90:329-348); lanes that left the chain are zeroed.  w overwrites y; partial dot w . w.
__device__ __forceinline__ void project_node(const OpView& op, int i, unsigned long long chimask, double2* x) {
  int s0 = op.stab_ptr[i], s1 = op.stab_ptr[i + 1];
  int ns = s1 - s0;
  if (ns <= 1) return;
  double2 acc[9];
  for (int l = 0; l < 9; ++l) acc[l] = make_double2(0, 0);
  for (int j = s0; j < s1; ++j) {
    int g = op.stab[j];
    bool neg = (chimask >> g) & 1ull;
    uint32_t sgm = op.sgm[g];
    for (int l = 0; l < 9; ++l) {
      double2 v = x[op.pi[g * 9 + l]];
      if (((sgm >> l) & 1u) ^ (neg ? 1u : 0u)) v = make_double2(-v.x, -v.y);
      acc[l] = cadd(acc[l], v);
    }
  }
  for (int l = 0; l < 9; ++l) x[l] = cscale(acc[l], 1.0 / (double)ns);
}

template <typename ST>
__global__ void __launch_bounds__(WPB * TL) k_lanczos_w(OpView op, BatchView bv, typename St2<ST>::T* __restrict__ y,
                                                        const typename St2<ST>::T* __restrict__ u,
                                                        const typename St2<ST>::T* __restrict__ up, double2* part, int npw) {
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
        x[l] = csub(csub(ld(y + q), cmul(as, ld(u + q))), cmul(bs, ld(up + q)));
      }
      if (bv.project) project_node(op, i, chim, x);
      for (int l = 0; l < 9; ++l) dot = cadd(dot, cmul(x[l], x[l]));
    } else {
      for (int l = 0; l < 9; ++l) x[l] = make_double2(0, 0);
    }
    for (int l = 0; l < 9; ++l) stv(y + vix(it.tile, bv.nn, i, l) + lane, x[l]);
  }
  block_reduce_store(dot, part, it.tile, bpt);
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
// a_k = sum of the partials (fixed order); depth test every 4 levels from 8 (src/asr_edc.f90:121-127)
__global__ void k_reduce_a(BatchView bv, const double2* part, int bpt, int k) {
  int tile = blockIdx.x, lane = threadIdx.x;
  if (tile >= bv.ntile || !bv.tile_act[tile]) return;
  int L = tile * TL + lane;
  int grp = bv.lane_group[L];
  bv.lane_wact[L] = 0;
  if (grp < 0 || !bv.lane_act[L]) return;
  double2 a = make_double2(0, 0);
  for (int q = 0; q < bpt; ++q) a = cadd(a, part[((size_t)tile * bpt + q) * TL + lane]);
  bv.acur[L] = a;
  bv.acoef[(size_t)L * NLMAX + k - 1] = a;
  bv.lane_m[L] = k;
  int nlev = bv.ginfo[grp].nlev;
  bool go = true;
  if (k == nlev) {
    go = false;   // edc exits before b_k (src/asr_edc.f90:120); the plain chain still forms b_n (asr_recursion.f90:50-57)
    if (bv.mode == ASR_MODE_PLAIN) bv.lane_wact[L] = 1;
  } else if (bv.depth_tol > 0.0 && k >= 8 && k % 4 == 0 && bv.mode == ASR_MODE_EDC) {
    double2 wd[NLMAX], we[NLMAX];
    int nf = 0;
    double2 gtry = cf_species_dev(bv.acoef + (size_t)L * NLMAX, bv.bcoef + (size_t)L * NLMAX, k, bv.lane_z[L], bv.tail, wd, we,
                                  &nf, nullptr);
    if (nf) atomicAdd(bv.nfall, nf);
    if (k > 8 && cabs2(csub(gtry, bv.gprev[L])) <= bv.depth_tol * cabs2(gtry)) go = false;
    bv.gprev[L] = gtry;
  }
  if (go) bv.lane_wact[L] = 1;
  else bv.lane_act[L] = 0;
}

// b_k = sqrt(w . w); |b| < tol ends the chain; scales of the next step (u <- w / b, up <- u)
__global__ void k_reduce_b(BatchView bv, const double2* part, int bpt, int k, double btol) {
  int tile = blockIdx.x, lane = threadIdx.x;
  if (tile >= bv.ntile) return;
  int L = tile * TL + lane;
  int grp = bv.lane_group[L];
  bool act = false;
  if (bv.tile_act[tile] && grp >= 0 && bv.lane_wact[L]) {
    double2 ww = make_double2(0, 0);
    for (int q = 0; q < bpt; ++q) ww = cadd(ww, part[((size_t)tile * bpt + q) * TL + lane]);
    double2 b = bv.mode == ASR_MODE_PLAIN ? make_double2(sqrt(ww.x), 0.0) : csqrt_p(ww);
    bv.bcoef[(size_t)L * NLMAX + k - 1] = b;
    bool ok = bv.mode == ASR_MODE_PLAIN ? (b.x >= btol) : (cabs2(b) >= btol);
    if (!bv.lane_act[L]) ok = false;   // plain chain at its last level: b_n stored, chain done
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

template <typename T>
struct Dev {
  T* p = nullptr;
  size_t n = 0;
  ~Dev() { if (p) cudaFree(p); }
  int alloc(size_t m) {
    if (m <= n && p) return ASR_OK;
    if (p) cudaFree(p);
    p = nullptr; n = 0;
    if (cudaMalloc(&p, std::max<size_t>(m, 1) * sizeof(T)) != cudaSuccess) {
      set_error("chains: device allocation of %zu bytes failed", m * sizeof(T));
      return ASR_ENOMEM;
    }
    n = m;
    return ASR_OK;
  }
};

size_t smul_smem(const asr_op* op, size_t st_size) {
  size_t b = (size_t)op->ntype * (op->nslot + 1) * 81 * st_size;
  b += (op->nop * 9 + 1) & ~1;
  b += op->nop * sizeof(uint16_t);
  b = (b + 15) & ~(size_t)15;
  b += TL * 9 * sizeof(double) + 16;
  return b;
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
    k_smul<ST, true, true><<<grid, B, sm, s>>>(ov, bv, blk, U, Y, part, npw);
    return ASR_OK;
  }
  // t1 = D x0, t2 = S t1
  if (all_dunif) {
    k_smul<ST, true, false><<<grid, B, sm, s>>>(ov, bv, blk, U, T2, part, npw);
  } else {
    k_rand<ST><<<grid, B, 0, s>>>(ov, bv, PD, U, true, T1, npw);
    k_smul<ST, false, false><<<grid, B, sm, s>>>(ov, bv, blk, T1, T2, part, npw);
  }
  if (!any_o) {   // y = s sq (D t2 + (c + e + X) x0)
    k_combine<ST><<<grid, B, 0, s>>>(ov, bv, T2, U, true, PCEB, true, U, false, nullptr, 1.0, true, Y, part, npw);
    return ASR_OK;
  }
  // h1 = D t2 + C x0;  r1 = O h1;  h2 = D S D r1 + C r1;  y = s sq (h1 - h2 + (e + X) x0)
  k_combine<ST><<<grid, B, 0, s>>>(ov, bv, T2, U, true, PC, false, U, false, nullptr, 1.0, false, H1, part, npw);
  k_rand<ST><<<grid, B, 0, s>>>(ov, bv, PO, H1, false, R1, npw);
  k_rand<ST><<<grid, B, 0, s>>>(ov, bv, PD, R1, false, T1, npw);   // t1 = D r1 (r1 is in amplitude coordinates)
  k_smul<ST, false, false><<<grid, B, sm, s>>>(ov, bv, blk, T1, T2, part, npw);
  k_combine<ST><<<grid, B, 0, s>>>(ov, bv, T2, R1, false, PC, false, U, true, H1, -1.0, true, Y, part, npw);
  return ASR_OK;
}

template <typename ST>
int run_lanes_t(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                const GroupLayout& GL, const std::vector<int>& lane_group, const double2* d_lane_z, int nlane,
                const RunOptions& opt, double2* d_g_out, std::vector<double2>* a_out, std::vector<double2>* b_out,
                std::vector<int>* m_out, int64_t* nfall_out, int64_t* nsteps_out) {
  typedef typename St2<ST>::T T2;
  cudaStream_t s = ctx->stream;
  const int nn = op->nn;
  const int ntile_all = (nlane + TL - 1) / TL;
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
  // batch size: tiles in flight bounded by memory (3 vectors + temporaries per tile) and by 8 tiles
  const size_t vec_bytes = (size_t)nn * 9 * TL * sizeof(T2);
  const int nvec = 3 + (fused ? 0 : (any_o ? 4 : 2));
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  int tpb = opt.tiles_per_batch > 0 ? opt.tiles_per_batch : 8;
  while (tpb > 1 && (size_t)tpb * nvec * vec_bytes > freeb / 2) tpb /= 2;
  tpb = std::min(tpb, ntile_all);
  const int npw = std::max(1, opt.nodes_per_warp);
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
  Dev<int> d_lgroup, d_act, d_wact, d_m, d_tact, d_nfall;
  Dev<double2> d_a, d_b, d_gprev, d_acur, d_bprev, d_su, d_sup, d_part, d_z;
  ASR_TRY(d_lgroup.alloc(nlp)); ASR_TRY(d_act.alloc(nlp)); ASR_TRY(d_wact.alloc(nlp)); ASR_TRY(d_m.alloc(nlp));
  ASR_TRY(d_tact.alloc(tpb)); ASR_TRY(d_nfall.alloc(1));
  ASR_TRY(d_a.alloc((size_t)nlp * NLMAX)); ASR_TRY(d_b.alloc((size_t)nlp * NLMAX));
  ASR_TRY(d_gprev.alloc(nlp)); ASR_TRY(d_acur.alloc(nlp)); ASR_TRY(d_bprev.alloc(nlp)); ASR_TRY(d_su.alloc(nlp));
  ASR_TRY(d_sup.alloc(nlp)); ASR_TRY(d_part.alloc((size_t)tpb * bpt * TL)); ASR_TRY(d_z.alloc(nlp));
  Dev<T2> V[7];
  for (int q = 0; q < nvec; ++q) ASR_TRY(V[q].alloc((size_t)tpb * nn * 9 * TL));
  ASR_CUDA(cudaMemsetAsync(d_nfall.p, 0, sizeof(int), s));
  if (a_out) { a_out->assign((size_t)nlane * NLMAX, make_double2(0, 0)); b_out->assign((size_t)nlane * NLMAX, make_double2(0, 0)); }
  if (m_out) m_out->assign(nlane, 0);
  std::vector<int> hgroup(nlp), lmap(nlp), hm_all(nlane, 0);
  std::vector<double2> ha, hb;
  Dev<int> d_lmap, d_m_all;
  ASR_TRY(d_lmap.alloc(nlp));
  ASR_TRY(d_m_all.alloc(nlane));
  ASR_CUDA(cudaMemsetAsync(d_m_all.p, 0, nlane * sizeof(int), s));
  // tiles of 32 consecutive lanes, deepest first, so that every batch runs to one depth
  std::vector<int> tdepth(ntile_all, 0), order(ntile_all);
  for (int L = 0; L < nlane; ++L) tdepth[L / TL] = std::max(tdepth[L / TL], ginfo[lane_group[L]].nlev);
  for (int t = 0; t < ntile_all; ++t) order[t] = t;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tdepth[x] > tdepth[y]; });
  std::vector<double2> one(nlp, make_double2(1.0, 0.0));
  for (int t0 = 0; t0 < ntile_all; t0 += tpb) {
    const int nt = std::min(tpb, ntile_all - t0);
    int kmax = 0;
    std::vector<int> tact(tpb, 0), ones(nlp, 0);
    for (int q = 0; q < nlp; ++q) {
      int bt = q / TL;
      int L = bt < nt ? order[t0 + bt] * TL + q % TL : -1;
      if (L >= nlane) L = -1;
      lmap[q] = L;
      hgroup[q] = L >= 0 ? lane_group[L] : -1;
      if (hgroup[q] >= 0) { kmax = std::max(kmax, ginfo[hgroup[q]].nlev); tact[bt] = 1; ones[q] = 1; }
    }
    ASR_CUDA(cudaMemcpyAsync(d_lgroup.p, hgroup.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_lmap.p, lmap.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_act.p, ones.data(), nlp * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemcpyAsync(d_tact.p, tact.data(), tpb * sizeof(int), cudaMemcpyHostToDevice, s));
    ASR_CUDA(cudaMemsetAsync(d_wact.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_m.p, 0, nlp * sizeof(int), s));
    ASR_CUDA(cudaMemsetAsync(d_a.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_b.p, 0, (size_t)nlp * NLMAX * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_gprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_bprev.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemsetAsync(d_sup.p, 0, nlp * sizeof(double2), s));
    ASR_CUDA(cudaMemcpyAsync(d_su.p, one.data(), nlp * sizeof(double2), cudaMemcpyHostToDevice, s));
    k_gather_z<<<(nlp + 127) / 128, 128, 0, s>>>(nlp, d_lmap.p, d_lane_z, d_z.p);
    BatchView bv{nt, nn, op->nsmax, 0, opt.mode, opt.project, opt.tail, NLMAX, opt.depth_tol, d_gblob.p, GL, d_ginfo.p,
                 d_lgroup.p, d_z.p, d_act.p, d_wact.p, d_m.p, d_a.p, d_b.p, d_gprev.p, d_acur.p, d_bprev.p, d_su.p, d_sup.p,
                 d_tact.p, d_nfall.p};
    k_init<ST><<<std::min<size_t>(65535, ((size_t)nt * nn * 9 * TL + 255) / 256), 256, 0, s>>>(bv, V[1].p, V[0].p);
    ctx->launches += 2;
    const int gridb = nt * bpt;
    if (ctx->profile) {   // event pairs stay pending until asr_ctx_kernel_stats reads them (no synchronisation here)
      while ((int)ctx->ev_pool.size() < 2 * (ctx->ev_used + kmax)) {
        cudaEvent_t e;
        ASR_CUDA(cudaEventCreate(&e));
        ctx->ev_pool.push_back(e);
      }
    }
    for (int k = 1; k <= kmax; ++k) {
      bv.kstep = k;
      T2* U = V[k % 3].p;
      T2* UP = V[(k + 2) % 3].p;
      T2* Y = V[(k + 1) % 3].p;
      if (ctx->profile) ASR_CUDA(cudaEventRecord(ctx->ev_pool[2 * ctx->ev_used], s));
      ASR_TRY(step_apply<ST>(ctx, op, bv, fused, any_o, all_dunif, U, Y, nvec > 3 ? V[3].p : nullptr, nvec > 3 ? V[4].p : nullptr,
                             nvec > 5 ? V[5].p : nullptr, nvec > 5 ? V[6].p : nullptr, d_part.p, npw, gridb));
      if (ctx->profile) {
        ASR_CUDA(cudaEventRecord(ctx->ev_pool[2 * ctx->ev_used + 1], s));
        ++ctx->ev_used;
        // algorithmic traffic of one operator pass: read U and write Y per (node, lane), plus the node tables per tile
        const double tab = (double)op->nslot * 5 + (double)op->nsmax * 5 + 8 + 8 + 4;
        ctx->prof_bytes += (double)nt * nn * (2.0 * 9 * TL * sizeof(T2) + tab);
        ctx->prof_flops += (double)nt * nn * TL * (op->nslot + 1) * 81.0 * 4.0;
        ctx->prof_launches += 1;
      }
      k_reduce_a<<<nt, TL, 0, s>>>(bv, d_part.p, bpt, k);
      k_lanczos_w<ST><<<gridb, WPB * TL, 0, s>>>(op->view(), bv, Y, U, UP, d_part.p, npw);
      k_reduce_b<<<nt, TL, 0, s>>>(bv, d_part.p, bpt, k, 1.0e-12);
      ctx->launches += 3 + (fused ? 1 : (any_o ? 7 : (all_dunif ? 2 : 3)));
    }
    ASR_CUDA(cudaGetLastError());
    if (opt.mode == ASR_MODE_EDC && d_g_out) {
      k_cf_final<<<(nlp + 63) / 64, 64, 0, s>>>(bv, nlp, d_lmap.p, d_g_out);
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
  ASR_CUDA(cudaMemcpyAsync(hm_all.data(), d_m_all.p, nlane * sizeof(int), cudaMemcpyDeviceToHost, s));
  int64_t nsteps = 0;
  int nf = 0;
  ASR_CUDA(cudaMemcpyAsync(&nf, d_nfall.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  for (int L = 0; L < nlane; ++L) nsteps += hm_all[L];
  if (m_out) *m_out = hm_all;
  if (nfall_out) *nfall_out = nf;
  if (nsteps_out) *nsteps_out = nsteps;
  return ASR_OK;
}

}  // namespace

int run_lanes(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
              const GroupLayout& GL, const std::vector<int>& lane_group, const double2* d_lane_z, int nlane,
              const RunOptions& opt, double2* d_g_out, std::vector<double2>* a_out, std::vector<double2>* b_out,
              std::vector<int>* m_out, int64_t* nfall_out, int64_t* nsteps_out) {
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_smul<double, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_smul<double, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_smul<double, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_smul<float, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_smul<float, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_smul<float, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    attr_done = true;
  }
  if (smul_smem(op, sizeof(double)) > 96 * 1024) { set_error("chains: bond tables above 96 KB of shared memory"); return ASR_EINVAL; }
  if (opt.precision == ASR_FP32)
    return run_lanes_t<float>(ctx, op, ginfo, gblob, GL, lane_group, d_lane_z, nlane, opt, d_g_out, a_out, b_out, m_out, nfall_out,
                              nsteps_out);
  return run_lanes_t<double>(ctx, op, ginfo, gblob, GL, lane_group, d_lane_z, nlane, opt, d_g_out, a_out, b_out, m_out, nfall_out,
                             nsteps_out);
}

// ------------------------------------------------------------------------------------------------ drop-in applications
int apply_vectors(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                  const GroupLayout& GL, int nvec, const double* x_host, bool complex_in, double* y_host, int what) {
  cudaStream_t s = ctx->stream;
  const int nn = op->nn;
  const int nt = (nvec + TL - 1) / TL;
  const size_t nel = (size_t)nt * nn * 9 * TL;
  std::vector<double2> hx(nel, make_double2(0, 0));
  for (int v = 0; v < nvec; ++v)
    for (int i = 0; i < nn; ++i)
      for (int l = 0; l < 9; ++l) {
        size_t src = (size_t)v * 9 * nn + 9 * (size_t)i + l;
        size_t dst = (((size_t)(v / TL) * nn + i) * 9 + l) * TL + v % TL;
        hx[dst] = complex_in ? make_double2(x_host[2 * src], x_host[2 * src + 1]) : make_double2(x_host[src], 0.0);
      }
  Dev<double> d_gblob;
  Dev<GroupInfo> d_ginfo;
  ASR_TRY(d_gblob.alloc(gblob.size()));
  ASR_TRY(d_ginfo.alloc(ginfo.size()));
  ASR_CUDA(cudaMemcpyAsync(d_gblob.p, gblob.data(), gblob.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_ginfo.p, ginfo.data(), ginfo.size() * sizeof(GroupInfo), cudaMemcpyHostToDevice, s));
  const int nlp = nt * TL;
  const int npw = 4, npb = WPB * npw, bpt = (nn + npb - 1) / npb;
  std::vector<int> hgroup(nlp), ones(nlp, 1), tact(nt, 1);
  for (int q = 0; q < nlp; ++q) hgroup[q] = q < nvec ? 0 : -1;
  std::vector<double2> hz(nlp, make_double2(0.0, what == APPLY_RAND_Z ? 1.0 : 0.0)), hsu(nlp, make_double2(1.0, 0.0));
  Dev<int> d_lgroup, d_act, d_tact;
  Dev<double2> d_z, d_su, d_part, V[6];
  ASR_TRY(d_lgroup.alloc(nlp)); ASR_TRY(d_act.alloc(nlp)); ASR_TRY(d_tact.alloc(nt)); ASR_TRY(d_z.alloc(nlp));
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
  bv.ginfo = d_ginfo.p; bv.lane_group = d_lgroup.p; bv.lane_z = d_z.p; bv.lane_act = d_act.p; bv.lane_wact = d_act.p;
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
    // w = sq X(x / sq) with X = z pa + pb, z = i: the complex parameter par = pb + i pa
    k_combine<double><<<grid, WPB * TL, 0, s>>>(ov, bv, nullptr, V[0].p, true, PB, true, V[0].p, false, nullptr, 1.0, true, V[1].p,
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
        size_t dst = (size_t)v * 9 * nn + 9 * (size_t)i + l;
        double2 val = hy[(((size_t)(v / TL) * nn + i) * 9 + l) * TL + v % TL];
        if (complex_in || what != APPLY_H) { y_host[2 * dst] = val.x; y_host[2 * dst + 1] = val.y; }
        else y_host[dst] = val.x;
      }
  return ASR_OK;
}

}  // namespace asrb
