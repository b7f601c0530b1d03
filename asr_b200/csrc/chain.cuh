// Batched Lanczos chains on the site-class operator: device data layout and the host driver interface.
#pragma once
#include "op.h"

namespace asrb {

constexpr int TL = 32;       // lanes (chains) per tile: one warp covers one node of a tile
constexpr int NLMAX = 128;   // longest chain held on the device
constexpr int MAXOP = 64;    // chi masks are 64-bit

// Parameter blob of one group (doubles): for p in {c, d, o, e, pa, pb, c+e+pb, e+pb}: local weights
// W_p[kap][k_own][k_flip][l] (nw = ncls * nsm * nsm * 9 each), then the raw parameters par_p[s][l] (np = 9 * nsp each).
// The last two are the combined diagonal terms of the final step, C + E + X(z) and E + X(z), with X(z) = z pa + pb.
enum { PC = 0, PD = 1, PO = 2, PE = 3, PA = 4, PB = 5, PCEB = 6, PEB = 7, NPAR = 8 };
struct GroupLayout {
  int nw, np, stride;
  __host__ __device__ int w(int p) const { return p * nw; }
  __host__ __device__ int raw(int p) const { return NPAR * nw + p * np; }
};

// group flags
enum { GF_D_UNIFORM = 1, GF_O_ZERO = 2, GF_E_ZERO = 4, GF_X_ZERO = 8 };

struct GroupInfo {
  int flags;
  int frozen_sp;          // species frozen on the start site (0: none)
  int l0;                 // start orbital 1..9
  int nlev;
  unsigned long long chimask;   // bit g set: chi(g) = -1
  double dd[9];           // uniform d per orbital (GF_D_UNIFORM)
};

// Epilogue of the adjoint's operator application (the fused step kernel applied to wbar_k with unit scales): instead of
// A wbar it stores ubar_k = A wbar_k + ca Y_k - cb wbar_k - cc wbar_{k+1} and the per-lane partial dots ubar_k . X_k.
struct AdjEpi {
  const void* yk;          // Y_k = A u_k of the forward
  const void* wbn;         // wbar_{k+1}
  const void* xk;          // X_k (unscaled)
  void* ubk;               // output ubar_k
  const double2* ca;       // per lane: 2 abar_k
  const double2* cb;       // a_k
  const double2* cc;       // b_k (0 at the lane's last level)
};

// One batch: ntile tiles x TL lanes.  Lane L = tile * TL + j.
struct BatchView {
  int ntile, nn, nsm, kstep, mode, project, tail, nlevmax;
  double depth_tol;
  const double* gblob;
  GroupLayout GL;
  const GroupInfo* ginfo;
  const int* lane_group;   // -1: idle lane
  const int* tile_group;   // the group of every lane of the tile (tiles hold one group)
  const double2* lane_z;
  int* lane_act;           // 1 active
  int* lane_wact;          // 1: the lane computes w / b this step
  int* lane_m;
  double2* acoef;          // [lane][NLMAX]
  double2* bcoef;
  double2* gprev;
  double2* acur;           // a_k of this step
  double2* bprev;          // b_{k-1}
  double2* su;             // scale of the current vector
  double2* sup;            // scale of the previous vector
  int* tile_act;           // tile has an active lane
  int* nfall;
  int* lane_closed;        // optional: 1 where |b| < 1e-12 ended the chain
  int* tick;               // optional (ntile): per-tile tickets; set, the step and Lanczos kernels reduce a and b in the
                           // epilogue of the tile's last block instead of separate reduction launches
  void* t2out;             // optional: the fused step kernel also stores t2 = S (d o U) (unscaled, the vector type of the
                           // batch) for the adjoint's parameter gradient
  AdjEpi adj;              // the adjoint epilogue's vectors and coefficients (read only by that instantiation)
};

struct RunOptions {
  int mode = ASR_MODE_EDC;
  double depth_tol = 0.0;
  int tail = ASR_TAIL_HULL;
  int precision = ASR_FP64;
  int project = 1;
  int tiles_per_batch = 0;   // 0: automatic (the operator's tuned value, else 16 in FP64 and 8 in FP32)
  int nodes_per_warp = 0;    // 0: automatic (the operator's tuned value, else 4)
};

// owning device buffer (freed on scope exit)
template <typename T>
struct Dev {
  T* p = nullptr;
  size_t n = 0;
  Dev() = default;
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  ~Dev() { if (p) cudaFree(p); }
  int alloc(size_t m) {
    if (m <= n && p) return ASR_OK;
    if (p) cudaFree(p);
    p = nullptr; n = 0;
    if (cudaMalloc(&p, (m > 0 ? m : 1) * sizeof(T)) != cudaSuccess) {
      set_error("chains: device allocation of %zu bytes failed", m * sizeof(T));
      return ASR_ENOMEM;
    }
    n = m;
    return ASR_OK;
  }
};

// Projections of every Lanczos vector on target states (edc_green_proj, src/asr_edc.f90:174-232), device arrays:
// tnode (nsm, nt) 0-based node (-1: none), tgop (nsm, nt) 0-based operation, tw (9, nsm, nt, ngroup) dressing weights;
// outputs gp, gp4 (9, nt) per output lane (complex), gp4 with the chain cut four steps earlier.
struct ProjSpec {
  int nt = 0, nsm = 1;
  const int* tnode = nullptr;
  const int* tgop = nullptr;
  const double* tw = nullptr;
  double2* gp = nullptr;
  double2* gp4 = nullptr;
};
struct ProjView {
  int nt, nsm, kcap;
  const int* tnode;
  const int* tgop;
  const double* tw;
  double2* cpr;    // [tile][k][t * 9 + l][lane]
  double2* gp;
  double2* gp4;
};

// Runs chains for lanes (group, z) on the operator; results per lane: g (energy of the lane), a, b (NLMAX each), m.
// proj (optional): the projections of edc_green_proj for every lane; dev_ms (optional): the device time of the batches,
// allocations excluded.
int run_lanes(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
              const GroupLayout& GL, const std::vector<int>& lane_group, const double2* d_lane_z, int nlane,
              const RunOptions& opt, double2* d_g_out, std::vector<double2>* a_out, std::vector<double2>* b_out,
              std::vector<int>* m_out, int64_t* nfall_out, int64_t* nsteps_out, const ProjSpec* proj = nullptr,
              double* dev_ms = nullptr);

// EPI block chains (epi_blocks, src/asr_epi.f90:639-663): v9 (9, ngroup) start vectors on the start node; lane kind 0 runs
// from s0 with the projection on |v> = h'|s0>, kind 1 from |v> / |v| with the projection on s0; per lane g, f, |v|, depth
int run_epi(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
            const GroupLayout& GL, const std::vector<double>& v9, const std::vector<int>& lane_group,
            const std::vector<int>& lane_kind, const std::vector<double2>& lane_z, int tail, int project, int precision,
            std::vector<double2>& g_out, std::vector<double2>& f_out, std::vector<double>& nv_out, std::vector<int>& m_out,
            int64_t* nfall_out);

// route ed3: two chains per (group, energy) (lane kind 0: from |a>, 1: from |v>); per lane g, the projection f, the start
// norms |a|, |v| and the depth
int run_ed3(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
            const GroupLayout& GL, const std::vector<double>& oc, const std::vector<int>& lane_group,
            const std::vector<int>& lane_kind, const std::vector<double2>& lane_z, double depth_tol, int tail, int project,
            int precision, std::vector<double2>& g_out, std::vector<double2>& f_out, std::vector<double>& na_out,
            std::vector<double>& nv_out, std::vector<int>& m_out, std::vector<double2>* a_out, std::vector<double2>* b_out,
            std::vector<double2>* c_out, int64_t* nfall_out);

// reverse mode: G per lane, the depth each lane used (the depth test stops it when depth_tol > 0) and the gradients
// sum_lanes w_L dG_L/dpar per group, kinds c, d, pa, o, e (e and pb share one derivative), each (9, nsp)
int run_adjoint(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                const GroupLayout& GL, const std::vector<int>& lane_group, const std::vector<double2>& lane_z,
                const std::vector<double2>& lane_w, double depth_tol, int tail, int project, int stride, int precision,
                std::vector<double2>& g_out, std::vector<int>& m_out, std::vector<double2>& grad_out);

// y = H x style applications of the operator's own parameters on nvec vectors (normalised coordinates)
int apply_vectors(asr_ctx* ctx, asr_op* op, const std::vector<GroupInfo>& ginfo, const std::vector<double>& gblob,
                  const GroupLayout& GL, int nvec, const double* x_host, bool complex_in, double* y_host, int what);
enum { APPLY_H = 0, APPLY_RAND_Z = 1, APPLY_PROJECT = 2 };

}  // namespace asrb
