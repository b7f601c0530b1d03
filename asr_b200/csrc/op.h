// Internal types of the asr_b200 library: context, operator (device node tables) and the kernel-side views.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.cuh"

struct asr_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;      // the stream every call runs on
  cudaStream_t own_stream = nullptr;  // created by asr_ctx_create
  int num_sms = 148;
  int64_t nchain = 0, nlev = 0, nfall = 0;
  int64_t launches = 0;   // kernels launched by this context
  int* d_err = nullptr;   // device error word
  // kernel timing (asr_ctx_profile): device time, launches and algorithmic work per kernel kind (ASR_KERNEL_*)
  struct ProfStat {
    double ms = 0.0, bytes = 0.0, flops = 0.0;
    int64_t launches = 0;
  };
  int profile = 0;
  ProfStat prof[ASR_KERNEL_KINDS];
  std::vector<cudaEvent_t> ev_pool;   // pairs (start, end) of the timed launches
  std::vector<int> ev_kind;           // kernel kind of every recorded pair
  int ev_used = 0;                    // pairs recorded and not yet read
  // starts a timed region on stream s (returns its pair index, -1 when profiling is off); regions may nest (a level of
  // the reverse sweep and its kernels); no synchronisation
  int prof_start(cudaStream_t s) {
    if (!profile) return -1;
    while ((int)ev_pool.size() < 2 * (ev_used + 1)) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
      ev_pool.push_back(e);
    }
    if ((int)ev_kind.size() < ev_used + 1) ev_kind.resize(ev_used + 1);
    if (cudaEventRecord(ev_pool[2 * ev_used], s) != cudaSuccess) return -1;
    ev_kind[ev_used] = -1;   // open until prof_stop
    return ev_used++;
  }
  // ends the region `slot` of prof_start as one launch of `kind` with the given algorithmic bytes and flops
  void prof_stop(cudaStream_t s, int slot, int kind, double bytes, double flops) {
    if (slot < 0 || slot >= ev_used || ev_kind[slot] != -1) return;
    if (cudaEventRecord(ev_pool[2 * slot + 1], s) != cudaSuccess) return;
    ev_kind[slot] = kind;
    prof[kind].bytes += bytes;
    prof[kind].flops += flops;
    prof[kind].launches += 1;
  }
  unsigned char* cf_scratch = nullptr;   // device address of asr_cf_eval_noalloc's static array (resolved on first use)
  // the adjoint's vector slab, kept between calls while ws_hold is set (asr_ctx_hold_workspace)
  int ws_hold = 0;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  void ws_release() {
    if (ws) cudaFree(ws);
    ws = nullptr;
    ws_bytes = 0;
  }
};

namespace asrb {

// Device view of the node tables, passed by value to the kernels.  Node indices are 0-based, -1 = absent link;
// operation indices 0-based.  Layouts follow the reference: flipr/flipg (nsmax, nn) and hopr/hopg (nslot, nn) with the
// state / slot index fastest, i.e. hopr[k + nslot * i].
struct OpView {
  int nn, nslot, nsmax, nop, ncls, nsp, ntype;
  const int* site;        // (nn) 1-based graph site
  const int8_t* lst;      // (nn) own local state
  const int8_t* ncl;      // (nn) 0-based class
  const int8_t* typ;      // (nn) 0-based site type (stype of the site)
  const int8_t* start;    // (nn) 1 if the node sits on the start site
  const int8_t* frozen;   // (nn) operator-level frozen species (0: none)
  const double* sq;       // (nn) sqrt(orbit size)
  const double* isq;      // (nn) 1 / sqrt(orbit size)
  const int* flipr;       // (nsmax, nn)
  const uint8_t* flipg;
  const int* hopr;        // (nslot, nn)
  const uint8_t* hopg;
  const int* stab_ptr;    // (nn + 1) 0-based offsets
  const uint8_t* stab;    // (nstab)
  const int8_t* nsc;      // (ncls) species per class
  const uint8_t* pi;      // (9, nop) 0-based orbital permutation: D(g)[pi(l), l] = sg(l)
  const uint16_t* sgm;    // (nop) bit l set: sg(l, g) = -1
};

}  // namespace asrb

struct asr_op {
  asr_ctx* ctx = nullptr;
  int nn = 0, nslot = 0, nsmax = 0, nop = 0, ncls = 0, nsp = 0, ntype = 1, nsite = 0, nstab = 0, start_site = 1;
  int start_l = 1;
  // batch shape chosen by asr_autotune per precision (index 0 FP64, 1 FP32); 0: the built-in defaults
  int tuned_tpb[2] = {0, 0}, tuned_npw[2] = {0, 0};
  int tuned_link[2] = {0, 0};             // 1: the step kernel's fixed-offset link gathers (chosen by asr_autotune)
  double tuned_link_ms[2][2] = {{-1.0, -1.0}, {-1.0, -1.0}};   // device ms of the general / fixed-offset step at the tuned shape
  // host copies of the model and group
  std::vector<int> nsc, spc;       // spc(ldspc, ncls)
  int ldspc = 1;
  std::vector<double> mt;          // (nsm, nsm, nsm, ncls)
  std::vector<int> pi;             // (9, nop) 1-based
  std::vector<double> sg, chi, dmat;
  std::vector<double> block;       // (9, 9, nslot, ntype) unrotated bond blocks
  std::vector<double> block0;      // (9, 9, ntype)
  std::vector<double> c, d, o, e;  // (9, nsp) current operator parameters
  std::vector<int8_t> frozen_h;    // (nn) operator-level frozen species
  // host copies of what a freeze reads (device node order), fetched from the device tables on the first freeze: the site,
  // the own local state and the number of flip links of every node, and the class of the start node
  std::vector<int> site_h;
  std::vector<int8_t> lst_h, nflip_h;
  int start_class = -1;
  // device node order: the tables live in a locality order (reverse Cuthill-McKee of the hop graph, start node first);
  // old_of_new[n] is the reference (build) index of device node n, new_of_old its inverse; empty: the build order
  std::vector<int> old_of_new, new_of_old;
  int dev_node(int old) const { return new_of_old.empty() ? old : new_of_old[old]; }
  int ref_node(int dev) const { return old_of_new.empty() ? dev : old_of_new[dev]; }
  // device tables
  int* d_site = nullptr;
  int* d_level = nullptr;
  int* d_orb = nullptr;
  int8_t *d_lst = nullptr, *d_ncl = nullptr, *d_typ = nullptr, *d_start = nullptr, *d_frozen = nullptr;
  double *d_sq = nullptr, *d_isq = nullptr;
  int *d_flipr = nullptr, *d_hopr = nullptr, *d_stab_ptr = nullptr;
  uint8_t *d_flipg = nullptr, *d_hopg = nullptr, *d_stab = nullptr;
  int8_t* d_nsc = nullptr;
  uint8_t* d_pi = nullptr;
  uint16_t* d_sgm = nullptr;
  double* d_blocks = nullptr;   // [t][kk][l][l'] kk = 0: on-site block, kk = 1 + slot
  float* d_blocks_f = nullptr;
  asrb::OpView view() const {
    return asrb::OpView{nn, nslot, nsmax, nop, ncls, nsp, ntype, d_site, d_lst, d_ncl, d_typ, d_start, d_frozen,
                        d_sq, d_isq, d_flipr, d_flipg, d_hopr, d_hopg, d_stab_ptr, d_stab, d_nsc, d_pi, d_sgm};
  }
};

namespace asrb {
// graph_build.cu
int build_operator(asr_ctx* ctx, int nsite, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* cls,
                   const int* perm, int nop, int start, int maxlevel, int maxrank, const int* flippable, const int* stype,
                   asr_op* op, const int* tsite = nullptr, int ntarget = 0, int* tnode = nullptr, int* tgop = nullptr);
// host helpers (capi.cu)
void class_mt(const double* conc, int nsc, int nsm, double* mt);
}  // namespace asrb
