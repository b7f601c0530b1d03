// C ABI of asr_b200 (declarations and reference citations in include/asr_b200.h).
#include <chrono>
#include <cstdarg>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cf.cuh"
#include "chain.cuh"
#include "op.h"

namespace asrb {

static thread_local std::string g_err;
void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}
const char* get_error() { return g_err.c_str(); }

// augn_basis + class_mt (src/asr_augcls.f90:73-91, :190-205): mt(l, k, j) = x_j phi_l(j) phi_k(j) on the species of
// non-zero weight
void class_mt(const double* conc, int nsc, int nsm, double* mt) {
  for (int q = 0; q < nsm * nsm * nsm; ++q) mt[q] = 0.0;
  std::vector<int> sup;
  for (int j = 0; j < nsc; ++j) if (conc[j] > 0.0) sup.push_back(j);
  int n = (int)sup.size();
  std::vector<double> x(n), phi((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) x[j] = conc[sup[j]];
  auto P = [&](int l, int s) -> double& { return phi[l + (size_t)n * s]; };
  for (int s = 0; s < n; ++s) P(0, s) = 1.0;
  for (int l = 1; l < n; ++l) {
    for (int s = 0; s < n; ++s) P(l, s) = (s == l - 1) ? 1.0 : 0.0;
    for (int pass = 0; pass < 2; ++pass)
      for (int m = 0; m < l; ++m) {
        double ip = 0.0;
        for (int s = 0; s < n; ++s) ip += x[s] * P(m, s) * P(l, s);
        for (int s = 0; s < n; ++s) P(l, s) -= ip * P(m, s);
      }
    double nr = 0.0;
    for (int s = 0; s < n; ++s) nr += x[s] * P(l, s) * P(l, s);
    nr = std::sqrt(nr);
    for (int s = 0; s < n; ++s) P(l, s) /= nr;
  }
  for (int l = 0; l < n; ++l)
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j) mt[l + nsm * (k + nsm * (size_t)sup[j])] = x[j] * P(l, j) * P(k, j);
}

namespace {

// local_weights (src/asr_augcls.f90:362-377) into the device layout W[kap][own][flip][l]
void weights(const asr_op* op, const double* par, double* W) {
  const int nsm = op->nsmax;
  for (int kap = 0; kap < op->ncls; ++kap)
    for (int kk = 0; kk < nsm; ++kk)
      for (int k = 0; k < nsm; ++k)
        for (int lam = 0; lam < 9; ++lam) {
          double w = 0.0;
          if (k < op->nsc[kap] && kk < op->nsc[kap])
            for (int s = 0; s < op->nsc[kap]; ++s)
              w += par[lam + 9 * (size_t)(op->spc[s + (size_t)op->ldspc * kap] - 1)] * op->mt[k + nsm * (kk + nsm * (s + (size_t)nsm * kap))];
          W[((kap * nsm + k) * nsm + kk) * 9 + lam] = w;
        }
}

GroupLayout layout(const asr_op* op) {
  GroupLayout GL;
  GL.nw = op->ncls * op->nsmax * op->nsmax * 9;
  GL.np = 9 * op->nsp;
  GL.stride = NPAR * (GL.nw + GL.np);
  return GL;
}

bool all_equal_species(const double* p, int nsp) {
  for (int s = 1; s < nsp; ++s)
    for (int l = 0; l < 9; ++l) if (p[l + 9 * s] != p[l]) return false;
  return true;
}
bool all_zero(const double* p, int n) {
  for (int q = 0; q < n; ++q) if (p[q] != 0.0) return false;
  return true;
}

// one group: parameters -> blob + info
int make_group_slots(const asr_op* op, const GroupLayout& GL, const double* const* P, int frozen_sp, int l0, int nlev,
                     const double* chi_override, double* blob, GroupInfo& gi);

int make_group(const asr_op* op, const GroupLayout& GL, const double* c, const double* d, const double* o, const double* e,
               const double* pa, const double* pb, int frozen_sp, int l0, int nlev, const double* chi_override, double* blob,
               GroupInfo& gi) {
  const int np = 9 * op->nsp;
  std::vector<double> zero(np, 0.0), ceb(np), eb(np);
  const double* P[NPAR];
  P[PC] = c; P[PD] = d; P[PO] = o ? o : zero.data(); P[PE] = e ? e : zero.data();
  P[PA] = pa ? pa : zero.data(); P[PB] = pb ? pb : zero.data();
  for (int q = 0; q < np; ++q) { ceb[q] = P[PC][q] + P[PE][q] + P[PB][q]; eb[q] = P[PE][q] + P[PB][q]; }
  P[PCEB] = ceb.data(); P[PEB] = eb.data();
  return make_group_slots(op, GL, P, frozen_sp, l0, nlev, chi_override, blob, gi);
}

// weights and flags of a group from the raw parameter arrays of every blob slot (9, nsp each)
int make_group_slots(const asr_op* op, const GroupLayout& GL, const double* const* P, int frozen_sp, int l0, int nlev,
                     const double* chi_override, double* blob, GroupInfo& gi) {
  const int np = 9 * op->nsp;
  for (int p = 0; p < NPAR; ++p) {
    weights(op, P[p], blob + GL.w(p));
    for (int q = 0; q < np; ++q) blob[GL.raw(p) + q] = P[p][q];
  }
  gi.flags = 0;
  // d uniform over the species and invariant under the orbital permutations of the group: D x = d o x with d
  // commuting with every link operation, so it folds into the bond blocks
  bool dinv = true;
  for (int g = 0; g < op->nop && dinv; ++g)
    for (int l = 0; l < 9; ++l)
      if (P[PD][op->pi[l + 9 * g] - 1] != P[PD][l]) { dinv = false; break; }
  if (all_equal_species(P[PD], op->nsp) && dinv) gi.flags |= GF_D_UNIFORM;
  if (all_zero(P[PO], np)) gi.flags |= GF_O_ZERO;
  if (all_zero(P[PE], np)) gi.flags |= GF_E_ZERO;
  if (all_zero(P[PA], np) && all_zero(P[PB], np)) gi.flags |= GF_X_ZERO;
  for (int l = 0; l < 9; ++l) gi.dd[l] = P[PD][l];
  if (frozen_sp < 0 || frozen_sp > op->nsp) { set_error("chain group: frozen species out of range"); return ASR_EINVAL; }
  gi.frozen_sp = frozen_sp;
  if (l0 < 1 || l0 > 9) { set_error("chain group: start orbital out of range"); return ASR_EINVAL; }
  gi.l0 = l0;
  gi.nlev = nlev;
  gi.chimask = 0ull;
  if (op->nop > MAXOP) { set_error("chain group: at most %d operations", MAXOP); return ASR_EINVAL; }
  for (int g = 0; g < op->nop; ++g) {
    double v;
    if (chi_override) v = chi_override[g];
    else {
      v = op->dmat[(l0 - 1) + 9 * ((l0 - 1) + 9 * (size_t)g)];
      if (std::fabs(std::fabs(v) - 1.0) > 1.0e-9) {   // augcls_set_start, src/asr_augcls.f90:113-115
        set_error("augcls_set_start: start orbital is not one-dimensional under the group");
        return ASR_EINVAL;
      }
    }
    if (v < 0) gi.chimask |= (1ull << g);
  }
  return ASR_OK;
}

int upload_tables(asr_op* op, const double* dmat, const double* block, int nsb, int ntb, const double* block0) {
  cudaStream_t s = op->ctx->stream;
  const int nop = op->nop, ns = op->nslot, nty = op->ntype;
  op->dmat.assign(dmat, dmat + 81 * (size_t)nop);
  op->pi.assign(9 * (size_t)nop, 0);
  op->sg.assign(9 * (size_t)nop, 0.0);
  std::vector<uint8_t> pi0(9 * (size_t)nop);
  std::vector<uint16_t> sgm(nop, 0);
  for (int g = 0; g < nop; ++g)   // orbital operation tables: D[pi(l), l] = sg(l)  (src/asr_augcls.f90:728-736)
    for (int l = 0; l < 9; ++l) {
      for (int jj = 0; jj < 9; ++jj) {
        double v = dmat[jj + 9 * (l + 9 * (size_t)g)];
        if (std::fabs(v) > 0.5) { op->pi[l + 9 * g] = jj + 1; op->sg[l + 9 * g] = v; }
      }
      if (op->pi[l + 9 * g] == 0) { set_error("build_augcls_operator: orbital operation is not monomial"); return ASR_EINVAL; }
      pi0[g * 9 + l] = (uint8_t)(op->pi[l + 9 * g] - 1);
      if (op->sg[l + 9 * g] < 0) sgm[g] |= (uint16_t)(1u << l);
    }
  if (nsb < ns) { set_error("build_augcls_operator: fewer bond blocks than neighbour slots"); return ASR_EINVAL; }
  if (ntb < nty) { set_error("build_augcls_operator: site type without a bond table"); return ASR_EINVAL; }
  // unrotated blocks [t][kk][l][l'] (kk = 0: on-site)
  std::vector<double> B((size_t)nty * (ns + 1) * 81, 0.0);
  for (int t = 0; t < nty; ++t) {
    for (int l = 0; l < 9; ++l)
      for (int lp = 0; lp < 9; ++lp) {
        if (block0) B[((size_t)t * (ns + 1)) * 81 + l * 9 + lp] = block0[l + 9 * (lp + 9 * (size_t)t)];
        for (int k = 0; k < ns; ++k)
          B[((size_t)t * (ns + 1) + k + 1) * 81 + l * 9 + lp] = block[l + 9 * (lp + 9 * (k + (size_t)nsb * t))];
      }
  }
  op->block.assign(B.begin(), B.end());
  std::vector<float> Bf(B.begin(), B.end());
  std::vector<int8_t> nsc8(op->ncls);
  for (int k = 0; k < op->ncls; ++k) nsc8[k] = (int8_t)op->nsc[k];
  ASR_CUDA(cudaMalloc(&op->d_blocks, B.size() * sizeof(double)));
  ASR_CUDA(cudaMalloc(&op->d_blocks_f, B.size() * sizeof(float)));
  ASR_CUDA(cudaMalloc(&op->d_pi, pi0.size()));
  ASR_CUDA(cudaMalloc(&op->d_sgm, sgm.size() * sizeof(uint16_t)));
  ASR_CUDA(cudaMalloc(&op->d_nsc, nsc8.size()));
  ASR_CUDA(cudaMemcpyAsync(op->d_blocks, B.data(), B.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(op->d_blocks_f, Bf.data(), Bf.size() * sizeof(float), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(op->d_pi, pi0.data(), pi0.size(), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(op->d_sgm, sgm.data(), sgm.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(op->d_nsc, nsc8.data(), nsc8.size(), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  return ASR_OK;
}

void free_op(asr_op* op) {
  void* ptrs[] = {op->d_site, op->d_level, op->d_orb, op->d_lst, op->d_ncl, op->d_typ, op->d_start, op->d_frozen, op->d_sq,
                  op->d_isq, op->d_flipr, op->d_hopr, op->d_stab_ptr, op->d_flipg, op->d_hopg, op->d_stab, op->d_nsc,
                  op->d_pi, op->d_sgm, op->d_blocks, op->d_blocks_f};
  for (void* p : ptrs) if (p) cudaFree(p);
  delete op;
}

}  // namespace
}  // namespace asrb

using namespace asrb;

extern "C" {

int asr_version(void) { return 100; }

int asr_last_error(char* buf, size_t n) {
  if (!buf || n == 0) return ASR_EINVAL;
  std::strncpy(buf, get_error(), n - 1);
  buf[n - 1] = 0;
  return ASR_OK;
}

int asr_ctx_create(int device, asr_ctx** out) {
  if (!out) { set_error("asr_ctx_create: null output"); return ASR_EINVAL; }
  *out = nullptr;
  int ndev = 0;
  ASR_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) { set_error("asr_ctx_create: device %d of %d", device, ndev); return ASR_EINVAL; }
  ASR_ON_DEVICE(device);
  asr_ctx* c = new asr_ctx();
  c->device = device;
  cudaDeviceProp prop;
  ASR_CUDA(cudaGetDeviceProperties(&prop, device));
  c->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess) {
    set_error("asr_ctx_create: stream / allocation failed");
    delete c;
    return ASR_ECUDA;
  }
  cudaMemset(c->d_err, 0, sizeof(int));
  c->stream = c->own_stream;
  *out = c;
  return ASR_OK;
}

int asr_ctx_destroy(asr_ctx* ctx) {
  if (!ctx) return ASR_OK;
  DeviceGuard dg;
  dg.set(ctx->device);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  if (ctx->d_err) cudaFree(ctx->d_err);
  ctx->ws_release();
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  delete ctx;
  return ASR_OK;
}

int asr_ctx_set_stream(asr_ctx* ctx, void* stream) {
  if (!ctx) { set_error("asr_ctx_set_stream: null context"); return ASR_EINVAL; }
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return ASR_OK;
}

static int drain_events(asr_ctx* ctx) {
  if (ctx->ev_used == 0) return ASR_OK;
  ASR_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int q = 0; q < ctx->ev_used; ++q) {
    if (ctx->ev_kind[q] < 0) continue;   // started and never stopped (an error path)
    float ms = 0.f;
    ASR_CUDA(cudaEventElapsedTime(&ms, ctx->ev_pool[2 * q], ctx->ev_pool[2 * q + 1]));
    ctx->prof[ctx->ev_kind[q]].ms += ms;
  }
  ctx->ev_used = 0;
  return ASR_OK;
}

int asr_ctx_profile(asr_ctx* ctx, int on) {
  if (!ctx) { set_error("asr_ctx_profile: null context"); return ASR_EINVAL; }
  ASR_TRY(drain_events(ctx));
  ctx->profile = on;
  if (on)
    for (auto& p : ctx->prof) p = asr_ctx::ProfStat();
  return ASR_OK;
}

int asr_ctx_hold_workspace(asr_ctx* ctx, int on) {
  if (!ctx) { set_error("asr_ctx_hold_workspace: null context"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  if (!on && ctx->ws) {
    ASR_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->ws_release();
  }
  ctx->ws_hold = on != 0;
  return ASR_OK;
}

int asr_ctx_launches(asr_ctx* ctx, int64_t* launches) {
  if (!ctx || !launches) { set_error("asr_ctx_launches: null argument"); return ASR_EINVAL; }
  *launches = ctx->launches;
  return ASR_OK;
}

int asr_ctx_kernel_stats_kind(asr_ctx* ctx, int kind, double* ms, int64_t* launches, double* bytes, double* flops) {
  if (!ctx) { set_error("asr_ctx_kernel_stats: null context"); return ASR_EINVAL; }
  if (kind < 0 || kind >= ASR_KERNEL_KINDS) { set_error("asr_ctx_kernel_stats_kind: kind %d", kind); return ASR_EINVAL; }
  ASR_TRY(drain_events(ctx));
  const asr_ctx::ProfStat& p = ctx->prof[kind];
  if (ms) *ms = p.ms;
  if (launches) *launches = p.launches;
  if (bytes) *bytes = p.bytes;
  if (flops) *flops = p.flops;
  return ASR_OK;
}

int asr_ctx_kernel_stats(asr_ctx* ctx, double* ms, int64_t* launches, double* bytes, double* flops) {
  return asr_ctx_kernel_stats_kind(ctx, ASR_KERNEL_STEP, ms, launches, bytes, flops);
}

int asr_ctx_sync(asr_ctx* ctx) {
  ASR_ON_DEVICE(ctx->device);
  ASR_CUDA(cudaStreamSynchronize(ctx->stream));
  return ASR_OK;
}

int asr_ctx_stats(const asr_ctx* ctx, int64_t* nchain, int64_t* nlev, int64_t* nfall) {
  if (nchain) *nchain = ctx->nchain;
  if (nlev) *nlev = ctx->nlev;
  if (nfall) *nfall = ctx->nfall;
  return ASR_OK;
}

static int op_build(asr_ctx* ctx, int nsite, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc, int ldspc,
                    const double* conc, int nsp, const int* cls, const int* perm, int nop, const double* dmat, int start,
                    int maxlevel, int maxrank, const int* flippable, const int* stype, const double* block, int nblock_slots,
                    int ntype_blocks, const double* block0, const int* tsite, int ntarget, int* tnode, int* tgop,
                    asr_op** out) {
  if (!ctx || !out || !nbr_ptr || !nbr || !nsc || !spc || !conc || !cls || !perm || !dmat || !block) {
    set_error("asr_op_build: null argument");
    return ASR_EINVAL;
  }
  *out = nullptr;
  if (nsite < 1 || ncls < 1 || nop < 1 || nsp < 1 || ldspc < 1) { set_error("asr_op_build: empty input"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  for (int k = 0; k < ncls; ++k) {
    if (nsc[k] < 1 || nsc[k] > ldspc) { set_error("asr_op_build: species count of class %d", k + 1); return ASR_EINVAL; }
    double sum = 0.0;
    for (int j = 0; j < nsc[k]; ++j) {
      int sp = spc[j + (size_t)ldspc * k];
      if (sp < 1 || sp > nsp) { set_error("asr_op_build: species index out of range"); return ASR_EINVAL; }
      if (conc[j + (size_t)ldspc * k] < 0.0) { set_error("asr_op_build: negative concentration"); return ASR_EINVAL; }
      sum += conc[j + (size_t)ldspc * k];
    }
    if (std::fabs(sum - 1.0) > 1.0e-8) { set_error("asr_op_build: concentrations of class %d do not sum to 1", k + 1); return ASR_EINVAL; }
  }
  for (int i = 0; i < nsite; ++i) if (cls[i] < 1 || cls[i] > ncls) { set_error("asr_op_build: site class out of range"); return ASR_EINVAL; }
  int nty = 1;
  if (stype) for (int i = 0; i < nsite; ++i) {
    if (stype[i] < 1) { set_error("build_augcls_operator: site type without a bond table"); return ASR_EINVAL; }
    nty = std::max(nty, stype[i]);
  }
  if (nty > ntype_blocks) { set_error("build_augcls_operator: site type without a bond table"); return ASR_EINVAL; }
  asr_op* op = new asr_op();
  op->ctx = ctx;
  op->nsp = nsp;
  op->ntype = nty;
  op->nsc.assign(nsc, nsc + ncls);
  op->ldspc = ldspc;
  op->spc.assign(spc, spc + (size_t)ldspc * ncls);
  int rc = build_operator(ctx, nsite, nbr_ptr, nbr, ncls, nsc, cls, perm, nop, start, maxlevel, maxrank, flippable, stype, op,
                          tsite, ntarget, tnode, tgop);
  if (rc != ASR_OK) { free_op(op); return rc; }
  const int nsm = op->nsmax;
  op->mt.assign((size_t)nsm * nsm * nsm * ncls, 0.0);
  for (int k = 0; k < ncls; ++k) class_mt(conc + (size_t)ldspc * k, nsc[k], nsm, &op->mt[(size_t)nsm * nsm * nsm * k]);
  rc = upload_tables(op, dmat, block, nblock_slots, ntype_blocks, block0);
  if (rc != ASR_OK) { free_op(op); return rc; }
  op->c.assign(9 * (size_t)nsp, 0.0); op->d = op->c; op->o = op->c; op->e = op->c;
  op->frozen_h.assign(op->nn, 0);
  op->chi.assign(nop, 1.0);
  op->start_l = 1;
  *out = op;
  return ASR_OK;
}

int asr_op_build(asr_ctx* ctx, int nsite, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc, int ldspc,
                 const double* conc, int nsp, const int* cls, const int* perm, int nop, const double* dmat, int start,
                 int maxlevel, int maxrank, const int* flippable, const int* stype, const double* block, int nblock_slots,
                 int ntype_blocks, const double* block0, asr_op** out) {
  return op_build(ctx, nsite, nbr_ptr, nbr, ncls, nsc, spc, ldspc, conc, nsp, cls, perm, nop, dmat, start, maxlevel, maxrank,
                  flippable, stype, block, nblock_slots, ntype_blocks, block0, nullptr, 0, nullptr, nullptr, out);
}

int asr_op_build_targets(asr_ctx* ctx, int nsite, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc,
                         int ldspc, const double* conc, int nsp, const int* cls, const int* perm, int nop, const double* dmat,
                         int start, int maxlevel, int maxrank, const int* flippable, const int* stype, const double* block,
                         int nblock_slots, int ntype_blocks, const double* block0, const int* tsite, int ntarget, int* tnode,
                         int* tgop, asr_op** out) {
  if (ntarget < 0 || (ntarget > 0 && (!tsite || !tnode || !tgop))) {
    set_error("asr_op_build_targets: tsite needs tnode and tgop");
    return ASR_EINVAL;
  }
  return op_build(ctx, nsite, nbr_ptr, nbr, ncls, nsc, spc, ldspc, conc, nsp, cls, perm, nop, dmat, start, maxlevel, maxrank,
                  flippable, stype, block, nblock_slots, ntype_blocks, block0, tsite, ntarget, tnode, tgop, out);
}

int asr_op_free(asr_op* op) {
  if (!op) return ASR_OK;
  DeviceGuard dg;
  dg.set(op->ctx->device);
  free_op(op);
  return ASR_OK;
}

int asr_op_dims(const asr_op* op, int* dims) {
  if (!op || !dims) { set_error("asr_op_dims: null argument"); return ASR_EINVAL; }
  dims[0] = op->nn; dims[1] = op->nslot; dims[2] = op->nsmax; dims[3] = op->nop; dims[4] = op->ncls; dims[5] = op->ntype;
  dims[6] = op->nstab; dims[7] = op->nsp;
  return ASR_OK;
}

int asr_op_export_tables(const asr_op* op, int* flipr, int* flipg, int* hopr, int* hopg, int* lst, int* site, int* ncl, int* level,
                         double* norb, double* sq, int* stab_ptr, int* stab) {
  if (!op) { set_error("asr_op_export_tables: null operator"); return ASR_EINVAL; }
  asr_ctx* ctx = op->ctx;
  ASR_ON_DEVICE(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t nn = op->nn, nsm = op->nsmax, ns = op->nslot;
  std::vector<int> fr(nsm * nn), hr(ns * nn), sp(nn + 1), st(nn), lv(nn), ob(nn);
  std::vector<uint8_t> fg(nsm * nn), hg(ns * nn), sb(std::max(op->nstab, 1));
  std::vector<int8_t> ls(nn), nc(nn);
  std::vector<double> sqv(nn);
  ASR_CUDA(cudaMemcpyAsync(fr.data(), op->d_flipr, fr.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(fg.data(), op->d_flipg, fg.size(), cudaMemcpyDeviceToHost, s));
  if (ns) {
    ASR_CUDA(cudaMemcpyAsync(hr.data(), op->d_hopr, hr.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    ASR_CUDA(cudaMemcpyAsync(hg.data(), op->d_hopg, hg.size(), cudaMemcpyDeviceToHost, s));
  }
  ASR_CUDA(cudaMemcpyAsync(sp.data(), op->d_stab_ptr, sp.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (op->nstab) ASR_CUDA(cudaMemcpyAsync(sb.data(), op->d_stab, op->nstab, cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(st.data(), op->d_site, nn * sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(lv.data(), op->d_level, nn * sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(ob.data(), op->d_orb, nn * sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(ls.data(), op->d_lst, nn, cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(nc.data(), op->d_ncl, nn, cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(sqv.data(), op->d_sq, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  // the device keeps the nodes in its locality order: back to the reference numbering (node i of the build)
  auto ref = [&](int dev) { return dev >= 0 ? op->ref_node(dev) : -1; };
  for (size_t i = 0; i < nn; ++i) {
    const size_t n = (size_t)op->dev_node((int)i);
    for (size_t k = 0; k < nsm; ++k) {
      if (flipr) flipr[k + nsm * i] = ref(fr[k + nsm * n]) + 1;    // -1 -> 0 (absent), 0-based -> 1-based
      if (flipg) flipg[k + nsm * i] = fg[k + nsm * n] + 1;
    }
    for (size_t k = 0; k < ns; ++k) {
      if (hopr) hopr[k + ns * i] = ref(hr[k + ns * n]) + 1;
      if (hopg) hopg[k + ns * i] = hg[k + ns * n] + 1;
    }
    if (lst) lst[i] = ls[n];
    if (site) site[i] = st[n];
    if (ncl) ncl[i] = nc[n] + 1;
    if (level) level[i] = lv[n];
    if (norb) norb[i] = (double)ob[n];
    if (sq) sq[i] = sqv[n];
  }
  int pos = 0;
  for (size_t i = 0; i < nn; ++i) {
    const int n = op->dev_node((int)i), len = sp[n + 1] - sp[n];
    if (stab_ptr) stab_ptr[i] = pos + 1;
    if (stab) for (int q = 0; q < len; ++q) stab[pos + q] = sb[sp[n] + q] + 1;
    pos += len;
  }
  if (stab_ptr) stab_ptr[nn] = pos + 1;
  return ASR_OK;
}

int asr_op_set_params(asr_op* op, const double* c, const double* d, const double* o, const double* e) {
  if (!op || !c || !d || !o || !e) { set_error("augcls_set_params: null argument"); return ASR_EINVAL; }
  size_t m = 9 * (size_t)op->nsp;
  op->c.assign(c, c + m); op->d.assign(d, d + m); op->o.assign(o, o + m); op->e.assign(e, e + m);
  return ASR_OK;
}

// the node tables of a freeze, copied to the host once per operator (they do not change after the build)
static int freeze_tables(asr_op* op) {
  if (!op->site_h.empty()) return ASR_OK;
  cudaStream_t s = op->ctx->stream;
  const size_t nn = op->nn, nsm = op->nsmax;
  std::vector<int> st(nn), fr(nsm * nn);
  std::vector<int8_t> ls(nn), nc(1);
  ASR_CUDA(cudaMemcpyAsync(st.data(), op->d_site, nn * sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(fr.data(), op->d_flipr, fr.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(ls.data(), op->d_lst, nn, cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(nc.data(), op->d_ncl, 1, cudaMemcpyDeviceToHost, s));   // device node 0 is the start node
  ASR_CUDA(cudaStreamSynchronize(s));
  std::vector<int8_t> nf(nn, 0);
  for (size_t i = 0; i < nn; ++i)
    for (size_t k = 0; k < nsm; ++k) if (fr[k + nsm * i] >= 0) ++nf[i];
  op->site_h.swap(st);
  op->lst_h.swap(ls);
  op->nflip_h.swap(nf);
  op->start_class = nc[0];
  return ASR_OK;
}

// sets the frozen species of every node on `site` (each must sit on a site that was not flippable: own state 0, at most
// one flip link) and uploads the frozen array on the operator's stream (no synchronisation)
static int freeze_nodes(asr_op* op, int site, int sp, const char* who, int* nfound) {
  ASR_TRY(freeze_tables(op));
  int n = 0;
  for (int i = 0; i < op->nn; ++i) {
    if (op->site_h[i] != site) continue;
    if (op->lst_h[i] != 0 || op->nflip_h[i] > 1) { set_error("%s: the frozen site was flippable", who); return ASR_EINVAL; }
    ++n;
  }
  for (int i = 0; i < op->nn; ++i)
    if (op->site_h[i] == site) op->frozen_h[i] = (int8_t)sp;
  if (nfound) *nfound = n;
  // a pageable source: the call returns once the bytes are staged, so the host array may change afterwards
  ASR_CUDA(cudaMemcpyAsync(op->d_frozen, op->frozen_h.data(), op->nn, cudaMemcpyHostToDevice, op->ctx->stream));
  return ASR_OK;
}

int asr_op_freeze_site(asr_op* op, int site, int sp) {
  if (!op) { set_error("augcls_freeze_site: null operator"); return ASR_EINVAL; }
  if (sp < 1 || sp > op->nsp) { set_error("augcls_freeze_site: species index out of range"); return ASR_EINVAL; }
  ASR_ON_DEVICE(op->ctx->device);
  ASR_TRY(freeze_tables(op));
  if (op->site_h[0] == site) {   // the start site: its species must belong to the start node's class (:133-134)
    const int kap = op->start_class;
    bool in = false;
    for (int k = 0; k < op->nsc[kap]; ++k) if (op->spc[k + (size_t)op->ldspc * kap] == sp) in = true;
    if (!in) { set_error("augcls_freeze_site: species not in the class of the frozen site"); return ASR_EINVAL; }
  }
  return freeze_nodes(op, site, sp, "augcls_freeze_site", nullptr);
}

int asr_op_freeze_any(asr_op* op, int site, int sp, int* nfound) {
  if (!op) { set_error("augcls_freeze_any: null operator"); return ASR_EINVAL; }
  if (sp < 1 || sp > op->nsp) { set_error("augcls_freeze_any: species index out of range"); return ASR_EINVAL; }
  ASR_ON_DEVICE(op->ctx->device);
  return freeze_nodes(op, site, sp, "augcls_freeze_any", nfound);
}

int asr_op_unfreeze(asr_op* op) {
  if (!op) { set_error("asr_op_unfreeze: null operator"); return ASR_EINVAL; }
  ASR_ON_DEVICE(op->ctx->device);
  std::fill(op->frozen_h.begin(), op->frozen_h.end(), 0);
  ASR_CUDA(cudaMemsetAsync(op->d_frozen, 0, op->nn, op->ctx->stream));
  return ASR_OK;
}

int asr_op_set_start(asr_op* op, int l0) {
  if (!op || l0 < 1 || l0 > 9) { set_error("augcls_set_start: start orbital out of range"); return ASR_EINVAL; }
  for (int g = 0; g < op->nop; ++g) {
    double v = op->dmat[(l0 - 1) + 9 * ((l0 - 1) + 9 * (size_t)g)];
    if (std::fabs(std::fabs(v) - 1.0) > 1.0e-9) {
      set_error("augcls_set_start: start orbital is not one-dimensional under the group");
      return ASR_EINVAL;
    }
  }
  op->start_l = l0;
  for (int g = 0; g < op->nop; ++g) op->chi[g] = op->dmat[(l0 - 1) + 9 * ((l0 - 1) + 9 * (size_t)g)] >= 0 ? 1.0 : -1.0;
  return ASR_OK;
}

int asr_op_set_chi(asr_op* op, const double* chi) {
  if (!op || !chi) { set_error("augcls_set_chi: null argument"); return ASR_EINVAL; }
  for (int g = 0; g < op->nop; ++g) {
    if (std::fabs(std::fabs(chi[g]) - 1.0) > 1.0e-12) { set_error("augcls_set_chi: characters must be +-1"); return ASR_EINVAL; }
    op->chi[g] = chi[g];
  }
  return ASR_OK;
}

int asr_op_set_class_conc(asr_op* op, int kap, const double* conc) {
  if (!op || !conc || kap < 1 || kap > op->ncls) { set_error("augcls_set_class_conc: class out of range"); return ASR_EINVAL; }
  int nsc = op->nsc[kap - 1];
  double s = 0.0;
  for (int k = 0; k < nsc; ++k) {
    if (conc[k] < 0.0) { set_error("augcls_set_class_conc: concentrations"); return ASR_EINVAL; }
    s += conc[k];
  }
  if (std::fabs(s - 1.0) > 1.0e-8) { set_error("augcls_set_class_conc: concentrations"); return ASR_EINVAL; }
  const int nsm = op->nsmax;
  class_mt(conc, nsc, nsm, &op->mt[(size_t)nsm * nsm * nsm * (kap - 1)]);
  return ASR_OK;
}

static int op_group(asr_op* op, const GroupLayout& GL, const double* pa, const double* pb, std::vector<double>& blob,
                    std::vector<GroupInfo>& gi) {
  blob.assign(GL.stride, 0.0);
  gi.resize(1);
  return make_group(op, GL, op->c.data(), op->d.data(), op->o.data(), op->e.data(), pa, pb, 0, op->start_l, 1, op->chi.data(),
                    blob.data(), gi[0]);
}

int asr_op_apply(asr_op* op, const double* x, double* y, int nvec) {
  if (!op || !x || !y || nvec < 1) { set_error("augcls_apply: bad argument"); return ASR_EINVAL; }
  ASR_ON_DEVICE(op->ctx->device);
  GroupLayout GL = layout(op);
  std::vector<double> blob;
  std::vector<GroupInfo> gi;
  ASR_TRY(op_group(op, GL, nullptr, nullptr, blob, gi));
  return apply_vectors(op->ctx, op, gi, blob, GL, nvec, x, false, y, APPLY_H);
}

int asr_op_hp_c(asr_op* op, const double* x, double* y, int nvec) {
  if (!op || !x || !y || nvec < 1) { set_error("augcls_hp_c: bad argument"); return ASR_EINVAL; }
  ASR_ON_DEVICE(op->ctx->device);
  GroupLayout GL = layout(op);
  // h = c + D S D: the operator's c and d with o = e = 0 (H = E_nu + h - h o h reduces to h)
  std::vector<double> blob(GL.stride, 0.0), zero((size_t)9 * op->nsp, 0.0);
  std::vector<GroupInfo> gi(1);
  ASR_TRY(make_group(op, GL, op->c.data(), op->d.data(), zero.data(), zero.data(), nullptr, nullptr, 0, op->start_l, 1,
                     op->chi.data(), blob.data(), gi[0]));
  return apply_vectors(op->ctx, op, gi, blob, GL, nvec, x, true, y, APPLY_H);
}

int asr_op_rand_c(asr_op* op, const double* par, const double* x, double* w, int nvec) {
  if (!op || !par || !x || !w || nvec < 1) { set_error("augcls_rand_c: bad argument"); return ASR_EINVAL; }
  ASR_ON_DEVICE(op->ctx->device);
  GroupLayout GL = layout(op);
  const int np = 9 * op->nsp;
  std::vector<double> pr(np), pim(np);
  for (int q = 0; q < np; ++q) { pr[q] = par[2 * q]; pim[q] = par[2 * q + 1]; }
  std::vector<double> blob;
  std::vector<GroupInfo> gi;
  ASR_TRY(op_group(op, GL, pim.data(), pr.data(), blob, gi));   // X(z) = z pa + pb at z = i
  return apply_vectors(op->ctx, op, gi, blob, GL, nvec, x, true, w, APPLY_RAND_Z);
}

int asr_op_project_c(asr_op* op, double* x, int nvec) {
  if (!op || !x || nvec < 1) { set_error("augcls_project_c: bad argument"); return ASR_EINVAL; }
  ASR_ON_DEVICE(op->ctx->device);
  GroupLayout GL = layout(op);
  std::vector<double> blob;
  std::vector<GroupInfo> gi;
  ASR_TRY(op_group(op, GL, nullptr, nullptr, blob, gi));
  return apply_vectors(op->ctx, op, gi, blob, GL, nvec, x, true, x, APPLY_PROJECT);
}

static int chains_common(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double2* d_z, int nz, int mode,
                         double depth_tol, int tail, int precision, int project, double2* d_g, double* a, double* b,
                         int* mused) {
  if (!ctx || !op || !groups || ngroup < 1 || nz < 0) { set_error("asr_chains_run: bad argument"); return ASR_EINVAL; }
  if (mode != ASR_MODE_PLAIN && mode != ASR_MODE_EDC) { set_error("asr_chains_run: unknown mode"); return ASR_EINVAL; }
  if (tail < 0 || tail > 3) { set_error("asr_chains_run: unknown tail"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  cudaStream_t s = ctx->stream;
  GroupLayout GL = layout(op);
  std::vector<double> blob((size_t)GL.stride * ngroup, 0.0);
  std::vector<GroupInfo> gi(ngroup);
  int nlevmax = 0;
  for (int q = 0; q < ngroup; ++q) {
    const asr_chain_group& G = groups[q];
    if (!G.c || !G.d) { set_error("asr_chains_run: group %d without c or d", q + 1); return ASR_EINVAL; }
    if (G.nlev < 1 || G.nlev > NLMAX) { set_error("asr_chains_run: depth %d out of range 1..%d", G.nlev, NLMAX); return ASR_EINVAL; }
    ASR_TRY(make_group(op, GL, G.c, G.d, G.o, G.e, mode == ASR_MODE_EDC ? G.pa : nullptr, mode == ASR_MODE_EDC ? G.pb : nullptr,
                       G.frozen_sp, G.start_orb, G.nlev, nullptr, blob.data() + (size_t)GL.stride * q, gi[q]));
    nlevmax = std::max(nlevmax, G.nlev);
  }
  RunOptions opt;
  opt.mode = mode;
  opt.depth_tol = mode == ASR_MODE_EDC ? depth_tol : 0.0;
  opt.tail = tail;
  opt.precision = precision;
  opt.project = project;
  std::vector<double2> ha, hb;
  std::vector<int> hm;
  int64_t nfall = 0, nsteps = 0;
  const bool want_ab = a || b || mode == ASR_MODE_PLAIN;
  if (mode == ASR_MODE_EDC) {
    const int nlane = ngroup * nz;
    std::vector<int> lg(nlane);
    for (int q = 0; q < ngroup; ++q)
      for (int j = 0; j < nz; ++j) lg[(size_t)q * nz + j] = q;
    Dev<double2> d_lz;
    ASR_TRY(d_lz.alloc(nlane));
    for (int q = 0; q < ngroup; ++q)
      ASR_CUDA(cudaMemcpyAsync(d_lz.p + (size_t)q * nz, d_z, nz * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    ASR_TRY(run_lanes(ctx, op, gi, blob, GL, lg, d_lz.p, nlane, opt, d_g, want_ab ? &ha : nullptr, want_ab ? &hb : nullptr, &hm,
                      &nfall, &nsteps));
    for (int L = 0; L < nlane; ++L) {
      if (mused) mused[L] = hm[L];
      for (int k = 0; k < nlevmax; ++k) {
        size_t dst = 2 * ((size_t)L * nlevmax + k);
        if (a) { a[dst] = ha[(size_t)L * NLMAX + k].x; a[dst + 1] = ha[(size_t)L * NLMAX + k].y; }
        if (b) { b[dst] = hb[(size_t)L * NLMAX + k].x; b[dst + 1] = hb[(size_t)L * NLMAX + k].y; }
      }
    }
    ctx->nchain += nlane;
  } else {
    // plain: one real chain per group, then the terminated fraction at every energy
    std::vector<int> lg(ngroup);
    for (int q = 0; q < ngroup; ++q) lg[q] = q;
    Dev<double2> d_lz;
    ASR_TRY(d_lz.alloc(ngroup));
    ASR_CUDA(cudaMemsetAsync(d_lz.p, 0, ngroup * sizeof(double2), s));
    ASR_TRY(run_lanes(ctx, op, gi, blob, GL, lg, d_lz.p, ngroup, opt, nullptr, &ha, &hb, &hm, &nfall, &nsteps));
    // plain lanczos returns n levels with b(n) (src/reference/asr_recursion.f90:57)
    std::vector<double> ra((size_t)ngroup * NLMAX), rb((size_t)ngroup * NLMAX);
    std::vector<int> rn(ngroup);
    for (int q = 0; q < ngroup; ++q) {
      rn[q] = hm[q];
      for (int k = 0; k < NLMAX; ++k) { ra[(size_t)q * NLMAX + k] = ha[(size_t)q * NLMAX + k].x; rb[(size_t)q * NLMAX + k] = hb[(size_t)q * NLMAX + k].x; }
      if (mused) for (int j = 0; j < nz; ++j) mused[(size_t)q * nz + j] = hm[q];
      for (int k = 0; k < nlevmax; ++k) {
        size_t dst = 2 * ((size_t)q * nlevmax + k);
        if (a) { a[dst] = ra[(size_t)q * NLMAX + k]; a[dst + 1] = 0.0; }
        if (b) { b[dst] = rb[(size_t)q * NLMAX + k]; b[dst + 1] = 0.0; }
      }
    }
    if (d_g && nz > 0) {
      Dev<double> d_a, d_b, d_ai, d_bi;   // freed on every return path
      Dev<int> d_n;
      ASR_TRY(d_a.alloc(ra.size())); ASR_TRY(d_b.alloc(rb.size())); ASR_TRY(d_ai.alloc(ngroup)); ASR_TRY(d_bi.alloc(ngroup));
      ASR_TRY(d_n.alloc(ngroup));
      ASR_CUDA(cudaMemcpyAsync(d_a.p, ra.data(), ra.size() * sizeof(double), cudaMemcpyHostToDevice, s));
      ASR_CUDA(cudaMemcpyAsync(d_b.p, rb.data(), rb.size() * sizeof(double), cudaMemcpyHostToDevice, s));
      ASR_CUDA(cudaMemcpyAsync(d_n.p, rn.data(), ngroup * sizeof(int), cudaMemcpyHostToDevice, s));
      if (tail == ASR_TAIL_HULL) {
        // the complex cf_species hull tail on the real chain
        std::vector<double2> ca((size_t)ngroup * NLMAX), cb((size_t)ngroup * NLMAX);
        for (size_t q = 0; q < ca.size(); ++q) { ca[q] = make_double2(ra[q], 0.0); cb[q] = make_double2(rb[q], 0.0); }
        Dev<double2> d_ca, d_cb, d_zz;
        Dev<int> d_nf;
        ASR_TRY(d_ca.alloc(ca.size())); ASR_TRY(d_cb.alloc(cb.size())); ASR_TRY(d_zz.alloc((size_t)nz * ngroup));
        ASR_TRY(d_nf.alloc(1));
        ASR_CUDA(cudaMemsetAsync(d_nf.p, 0, sizeof(int), s));
        ASR_CUDA(cudaMemcpyAsync(d_ca.p, ca.data(), ca.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
        ASR_CUDA(cudaMemcpyAsync(d_cb.p, cb.data(), cb.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
        for (int q = 0; q < ngroup; ++q)
          ASR_CUDA(cudaMemcpyAsync(d_zz.p + (size_t)q * nz, d_z, nz * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        long nt = (long)nz * ngroup;
        k_cf_eval<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(d_ca.p, d_cb.p, d_n.p, NLMAX, ngroup, d_zz.p, nz, tail, d_g, nullptr,
                                                               d_nf.p);
        ASR_CUDA(cudaGetLastError());
        ASR_CUDA(cudaStreamSynchronize(s));
      } else {
        k_real_tail<<<(ngroup + 63) / 64, 64, 0, s>>>(d_a.p, d_b.p, d_n.p, NLMAX, ngroup, tail, d_ai.p, d_bi.p);
        long nt = (long)nz * ngroup;
        k_real_green<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(d_a.p, d_b.p, d_n.p, NLMAX, ngroup, d_ai.p, d_bi.p, tail, d_z, nz,
                                                                   d_g);
        ASR_CUDA(cudaGetLastError());
        ASR_CUDA(cudaStreamSynchronize(s));
      }
    }
    ctx->nchain += ngroup;
  }
  ctx->nlev += nsteps;
  ctx->nfall += nfall;
  return ASR_OK;
}

// epi_blocks (src/asr_epi.f90:639-663) for every (group, energy): v9 (9, ngroup) symmetry-adapted start vectors on the
// start node, chi (nop, ngroup) their characters (+-1); the chains of the edc route from s0 (projection on h'|s0>) and from
// h'|s0> / |h'|s0>| (projection on s0), full depth.  x (4, nz, ngroup) complex = X0, X1 (mean of the two chains), X2, and
// the X1 mismatch; mused (2, nz, ngroup) optional.
int asr_epi_blocks(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, const double* v9, const double* chi, int ngroup,
                   const double* z, int nz, int tail, int precision, int project, double* x, int* mused) {
  if (!ctx || !op || !groups || !v9 || !chi || ngroup < 1 || nz < 1 || !z || !x) { set_error("asr_epi_blocks: bad argument"); return ASR_EINVAL; }
  if (tail < 0 || tail > 3) { set_error("asr_epi_blocks: unknown tail"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  GroupLayout GL = layout(op);
  std::vector<double> blob((size_t)GL.stride * ngroup, 0.0), vv(9 * (size_t)ngroup);
  std::vector<GroupInfo> gi(ngroup);
  for (int q = 0; q < ngroup; ++q) {
    const asr_chain_group& G = groups[q];
    if (!G.c || !G.d || !G.pa || !G.pb) { set_error("asr_epi_blocks: group %d without c, d, pa or pb", q + 1); return ASR_EINVAL; }
    if (G.nlev < 1 || G.nlev > NLMAX) { set_error("asr_epi_blocks: depth %d out of range 1..%d", G.nlev, NLMAX); return ASR_EINVAL; }
    const double* cq = chi + (size_t)op->nop * q;
    for (int g = 0; g < op->nop; ++g)
      if (std::fabs(std::fabs(cq[g]) - 1.0) > 1.0e-12) { set_error("asr_epi_blocks: characters must be +-1"); return ASR_EINVAL; }
    double n2 = 0.0;
    for (int l = 0; l < 9; ++l) { vv[9 * (size_t)q + l] = v9[9 * (size_t)q + l]; n2 += v9[9 * (size_t)q + l] * v9[9 * (size_t)q + l]; }
    if (std::fabs(n2 - 1.0) > 1.0e-10) { set_error("asr_epi_blocks: start vector %d is not normalised", q + 1); return ASR_EINVAL; }
    ASR_TRY(make_group(op, GL, G.c, G.d, G.o, G.e, G.pa, G.pb, G.frozen_sp, G.start_orb, G.nlev, cq,
                       blob.data() + (size_t)GL.stride * q, gi[q]));
  }
  const int nlane = 2 * ngroup * nz;
  std::vector<int> lg(nlane), lk(nlane);
  std::vector<double2> lz(nlane);
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nz; ++j)
      for (int kd = 0; kd < 2; ++kd) {
        size_t L = 2 * ((size_t)q * nz + j) + kd;
        lg[L] = q; lk[L] = kd; lz[L] = make_double2(z[2 * j], z[2 * j + 1]);
      }
  std::vector<double2> g, f;
  std::vector<double> nv;
  std::vector<int> m;
  int64_t nfall = 0;
  ASR_TRY(run_epi(ctx, op, gi, blob, GL, vv, lg, lk, lz, tail, project, precision, g, f, nv, m, &nfall));
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nz; ++j) {
      size_t LU = 2 * ((size_t)q * nz + j), LV = LU + 1;
      double2 fa = f[LU], fb = cscale(f[LV], nv[LV]);
      double2 out[4] = {g[LU], cscale(cadd(fa, fb), 0.5), cscale(g[LV], nv[LV] * nv[LV]), csub(fa, fb)};
      for (int k = 0; k < 4; ++k) {
        size_t dst = 2 * (4 * ((size_t)j + (size_t)nz * q) + k);
        x[dst] = out[k].x;
        x[dst + 1] = out[k].y;
      }
      if (mused) { mused[2 * ((size_t)j + (size_t)nz * q)] = m[LU]; mused[2 * ((size_t)j + (size_t)nz * q) + 1] = m[LV]; }
    }
  ctx->nchain += nlane;
  ctx->nfall += nfall;
  return ASR_OK;
}

int asr_ed3_blocks(asr_ctx* ctx, asr_op* op, const asr_ed3_group* groups, int ngroup, const double* z, int nz, double depth_tol,
                   int tail, int precision, int project, double* bk, int* mused, double* a, double* b, double* c) {
  if (!ctx || !op || !groups || ngroup < 1 || nz < 1 || !z || !bk) { set_error("asr_ed3_blocks: bad argument"); return ASR_EINVAL; }
  if (tail < 0 || tail > 3) { set_error("asr_ed3_blocks: unknown tail"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  const int nsp = op->nsp, np = 9 * nsp;
  GroupLayout GL = layout(op);
  std::vector<double> blob((size_t)GL.stride * ngroup, 0.0), oc(ngroup);
  std::vector<GroupInfo> gi(ngroup);
  int nlevmax = 0;
  for (int q = 0; q < ngroup; ++q) {
    const asr_ed3_group& G = groups[q];
    if (!G.g || !G.d || !G.dc || !G.del || !G.enu || !G.o || !G.p) { set_error("asr_ed3_blocks: group %d incomplete", q + 1); return ASR_EINVAL; }
    if (G.nlev < 1 || G.nlev > NLMAX) { set_error("asr_ed3_blocks: depth %d out of range 1..%d", G.nlev, NLMAX); return ASR_EINVAL; }
    if (G.central < 1 || G.central > nsp) { set_error("asr_ed3_blocks: central species out of range"); return ASR_EINVAL; }
    if (G.start_orb < 1 || G.start_orb > 9) { set_error("asr_ed3_blocks: start orbital out of range"); return ASR_EINVAL; }
    // ed3_coefs (:91-107) as z-linear coefficients (the cf of ed3_blocks_blk, :281-288): et = z ea + eb, u = z ua + ub,
    // Qt = z qa + qb
    std::vector<double> ea(np), eb(np), ua(np), ub(np), qa(np), qb(np);
    for (int sp = 0; sp < nsp; ++sp)
      for (int l = 0; l < 9; ++l) {
        int k = l + 9 * sp;
        double r = G.dc[l] / G.del[k];
        ea[k] = r; eb[k] = -r * G.enu[k];
        ua[k] = G.o[k]; ub[k] = -G.o[k] * G.enu[k];
        qa[k] = -G.p[k] / r; qb[k] = (G.o[k] + G.p[k] * G.enu[k]) / r;
      }
    const double* P[NPAR];
    P[PC] = G.g; P[PD] = G.d; P[PO] = ea.data(); P[PE] = eb.data(); P[PA] = ua.data(); P[PB] = ub.data();
    P[PCEB] = qa.data(); P[PEB] = qb.data();
    ASR_TRY(make_group_slots(op, GL, P, G.central, G.start_orb, G.nlev, nullptr, blob.data() + (size_t)GL.stride * q, gi[q]));
    oc[q] = G.o[(G.start_orb - 1) + 9 * (size_t)(G.central - 1)];
    nlevmax = std::max(nlevmax, G.nlev);
  }
  const int nlane = 2 * ngroup * nz;
  std::vector<int> lg(nlane), lk(nlane);
  std::vector<double2> lz(nlane);
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nz; ++j)
      for (int kd = 0; kd < 2; ++kd) {
        size_t L = 2 * ((size_t)q * nz + j) + kd;
        lg[L] = q; lk[L] = kd; lz[L] = make_double2(z[2 * j], z[2 * j + 1]);
      }
  std::vector<double2> g, f, ha, hb, hc;
  std::vector<double> na, nv;
  std::vector<int> m;
  int64_t nfall = 0;
  int rc = run_ed3(ctx, op, gi, blob, GL, oc, lg, lk, lz, depth_tol, tail, project, precision, g, f, na, nv, m, a ? &ha : nullptr,
                   b ? &hb : nullptr, c ? &hc : nullptr, &nfall);
  if (rc != ASR_OK) return rc;
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nz; ++j) {
      size_t LA = 2 * ((size_t)q * nz + j), LV = LA + 1;
      double2 q0 = cscale(g[LA], na[LA] * na[LA]), q1a = cscale(f[LA], na[LA]);
      double2 q2 = cscale(g[LV], nv[LV] * nv[LV]), q1b = cscale(f[LV], nv[LV]);
      double2 fm = cscale(cadd(q1a, q1b), 0.5);
      double o = oc[q];
      double2 out[4] = {cadd(csub(q0, cscale(fm, 2.0 * o)), cscale(q2, o * o)), csub(fm, cscale(q2, o)), q2, csub(q1a, q1b)};
      for (int k = 0; k < 4; ++k) {
        size_t dst = 2 * (4 * ((size_t)j + (size_t)nz * q) + k);
        bk[dst] = out[k].x;
        bk[dst + 1] = out[k].y;
      }
      if (mused) { mused[2 * (j + (size_t)nz * q)] = m[LA]; mused[2 * (j + (size_t)nz * q) + 1] = m[LV]; }
      for (int kd = 0; kd < 2; ++kd)
        for (int k = 0; k < nlevmax; ++k) {
          size_t src = (LA + kd) * NLMAX + k, dst = 2 * ((LA + kd) * nlevmax + k);
          if (a) { a[dst] = ha[src].x; a[dst + 1] = ha[src].y; }
          if (b) { b[dst] = hb[src].x; b[dst + 1] = hb[src].y; }
          if (c) { c[dst] = hc[src].x; c[dst + 1] = hc[src].y; }
        }
    }
  ctx->nchain += nlane;
  ctx->nfall += nfall;
  return ASR_OK;
}

// the adjoint of the edc chains for every (group, energy) lane; grad receives nkind kinds (the first nkind of c, d, pa,
// o, e), symmetrised over the orbits of the orbitals under the point group
static int chains_adjoint_common(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz,
                                 const double* w, double depth_tol, int tail, int precision, int project, int stride,
                                 double* g, int* mused, double* grad, int nkind, const char* who) {
  if (!ctx || !op || !groups || ngroup < 1 || nz < 1 || !z || !w || !grad) { set_error("%s: bad argument", who); return ASR_EINVAL; }
  if (tail < ASR_TAIL_NONE || tail > ASR_TAIL_AVG2) { set_error("%s: unknown tail", who); return ASR_EINVAL; }
  if (depth_tol < 0.0) { set_error("%s: depth_tol must be >= 0", who); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  GroupLayout GL = layout(op);
  std::vector<double> blob((size_t)GL.stride * ngroup, 0.0);
  std::vector<GroupInfo> gi(ngroup);
  for (int q = 0; q < ngroup; ++q) {
    const asr_chain_group& G = groups[q];
    if (!G.c || !G.d || !G.pa || !G.pb) { set_error("%s: group %d needs c, d, pa, pb", who, q + 1); return ASR_EINVAL; }
    if (G.nlev < 1 || G.nlev > NLMAX) { set_error("%s: depth %d out of range 1..%d", who, G.nlev, NLMAX); return ASR_EINVAL; }
    ASR_TRY(make_group(op, GL, G.c, G.d, G.o, G.e, G.pa, G.pb, G.frozen_sp, G.start_orb, G.nlev, nullptr,
                       blob.data() + (size_t)GL.stride * q, gi[q]));
    if (nkind < 5 && !(gi[q].flags & GF_O_ZERO)) {
      set_error("%s: group %d has o != 0; asr_chains_adjoint_ext differentiates that operator", who, q + 1);
      return ASR_EINVAL;
    }
  }
  const int nlane = ngroup * nz;
  std::vector<int> lg(nlane), hm;
  std::vector<double2> lz(nlane), lw(nlane), hg, hgrad;
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nz; ++j) {
      size_t L = (size_t)q * nz + j;
      lg[L] = q;
      lz[L] = make_double2(z[2 * j], z[2 * j + 1]);
      lw[L] = make_double2(w[2 * L], w[2 * L + 1]);
    }
  int rc = run_adjoint(ctx, op, gi, blob, GL, lg, lz, lw, depth_tol, tail, project, stride, precision, hg, hm, hgrad);
  if (rc != ASR_OK) return rc;
  if (g)
    for (int L = 0; L < nlane; ++L) { g[2 * L] = hg[L].x; g[2 * L + 1] = hg[L].y; }
  if (mused) for (int L = 0; L < nlane; ++L) mused[L] = hm[L];
  const int nsp = op->nsp, nk = 5;
  // orbits of the orbitals under the point group (pi of every operation): the group-reduced operator represents
  // only parameters that are constant on each orbit, so the gradient is reported symmetrised over the orbits -- exact
  // along every invariant direction (per l, per irreducible orbit), while the single orbitals of a degenerate orbit are
  // not independent parameters
  std::vector<int> orbit(9);
  for (int l = 0; l < 9; ++l) orbit[l] = l;
  for (bool changed = true; changed;) {
    changed = false;
    for (int gop = 0; gop < op->nop; ++gop)
      for (int l = 0; l < 9; ++l) {
        int m = op->pi[l + 9 * gop] - 1, r = std::min(orbit[l], orbit[m]);
        if (orbit[l] != r || orbit[m] != r) { orbit[l] = orbit[m] = r; changed = true; }
      }
  }
  for (int q = 0; q < ngroup; ++q)
    for (int kind = 0; kind < nkind; ++kind)
      for (int sp = 0; sp < nsp; ++sp)
        for (int l = 0; l < 9; ++l) {
          double2 acc = make_double2(0, 0);
          int cnt = 0;
          for (int l2 = 0; l2 < 9; ++l2)
            if (orbit[l2] == orbit[l]) { acc = cadd(acc, hgrad[(((size_t)q * nk + kind) * 9 + l2) * nsp + sp]); ++cnt; }
          double2 v = cscale(acc, 1.0 / cnt);
          size_t dst = 2 * (l + 9 * (sp + (size_t)nsp * (kind + (size_t)nkind * q)));
          grad[dst] = v.x;
          grad[dst + 1] = v.y;
        }
  ctx->nchain += nlane;
  return ASR_OK;
}

int asr_chains_adjoint(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz,
                       const double* w, int tail, int precision, int project, int stride, double* g, double* grad) {
  return chains_adjoint_common(ctx, op, groups, ngroup, z, nz, w, 0.0, tail, precision, project, stride, g, nullptr, grad, 3,
                               "asr_chains_adjoint");
}

int asr_chains_adjoint_ext(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz,
                           const double* w, double depth_tol, int tail, int precision, int project, int stride, double* g,
                           int* mused, double* grad) {
  return chains_adjoint_common(ctx, op, groups, ngroup, z, nz, w, depth_tol, tail, precision, project, stride, g, mused, grad, 5,
                               "asr_chains_adjoint_ext");
}

// chain_worker tasks as explicit lanes (edc route): lane L runs group lane_group[L] (1-based) at the energy lane_z[L]
static int lanes_common(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const int* lane_group,
                        const double2* d_lane_z, int nlane, double depth_tol, int tail, int precision, int project, double2* d_g,
                        int* mused) {
  if (!ctx || !op || !groups || ngroup < 1 || !lane_group || nlane < 1) { set_error("asr_chains_run_lanes: bad argument"); return ASR_EINVAL; }
  if (tail < 0 || tail > 3) { set_error("asr_chains_run_lanes: unknown tail"); return ASR_EINVAL; }
  std::vector<int> lg(nlane);
  for (int L = 0; L < nlane; ++L) {
    if (lane_group[L] < 1 || lane_group[L] > ngroup) { set_error("asr_chains_run_lanes: lane %d has group %d", L + 1, lane_group[L]); return ASR_EINVAL; }
    lg[L] = lane_group[L] - 1;
  }
  ASR_ON_DEVICE(ctx->device);
  GroupLayout GL = layout(op);
  std::vector<double> blob((size_t)GL.stride * ngroup, 0.0);
  std::vector<GroupInfo> gi(ngroup);
  for (int q = 0; q < ngroup; ++q) {
    const asr_chain_group& G = groups[q];
    if (!G.c || !G.d) { set_error("asr_chains_run_lanes: group %d without c or d", q + 1); return ASR_EINVAL; }
    if (G.nlev < 1 || G.nlev > NLMAX) { set_error("asr_chains_run_lanes: depth %d out of range 1..%d", G.nlev, NLMAX); return ASR_EINVAL; }
    ASR_TRY(make_group(op, GL, G.c, G.d, G.o, G.e, G.pa, G.pb, G.frozen_sp, G.start_orb, G.nlev, nullptr,
                       blob.data() + (size_t)GL.stride * q, gi[q]));
  }
  RunOptions opt;
  opt.mode = ASR_MODE_EDC;
  opt.depth_tol = depth_tol;
  opt.tail = tail;
  opt.precision = precision;
  opt.project = project;
  std::vector<int> hm;
  int64_t nfall = 0, nsteps = 0;
  ASR_TRY(run_lanes(ctx, op, gi, blob, GL, lg, d_lane_z, nlane, opt, d_g, nullptr, nullptr, &hm, &nfall, &nsteps));
  if (mused) for (int L = 0; L < nlane; ++L) mused[L] = hm[L];
  ctx->nchain += nlane;
  ctx->nlev += nsteps;
  ctx->nfall += nfall;
  return ASR_OK;
}

int asr_chains_run_lanes(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const int* lane_group,
                         const double* lane_z, int nlane, double depth_tol, int tail, int precision, int project, double* g,
                         int* mused) {
  if (!ctx || !lane_z || !g || nlane < 1) { set_error("asr_chains_run_lanes: bad argument"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  cudaStream_t s = ctx->stream;
  Dev<double2> d_z, d_g;
  ASR_TRY(d_z.alloc(nlane));
  ASR_TRY(d_g.alloc(nlane));
  ASR_CUDA(cudaMemcpyAsync(d_z.p, lane_z, nlane * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_TRY(lanes_common(ctx, op, groups, ngroup, lane_group, d_z.p, nlane, depth_tol, tail, precision, project, d_g.p, mused));
  ASR_CUDA(cudaMemcpyAsync(g, d_g.p, nlane * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  return ASR_OK;
}

int asr_chains_run_lanes_dev(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const int* lane_group,
                             const void* lane_z_dev, int nlane, double depth_tol, int tail, int precision, int project,
                             void* g_dev) {
  if (!lane_z_dev || !g_dev) { set_error("asr_chains_run_lanes_dev: null device array"); return ASR_EINVAL; }
  return lanes_common(ctx, op, groups, ngroup, lane_group, (const double2*)lane_z_dev, nlane, depth_tol, tail, precision,
                      project, (double2*)g_dev, nullptr);
}

int asr_chains_run_dev(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const void* z_dev, int nz, int mode,
                       double depth_tol, int tail, int precision, int project, void* g_dev, double* a, double* b, int* mused) {
  return chains_common(ctx, op, groups, ngroup, (const double2*)z_dev, nz, mode, depth_tol, tail, precision, project,
                       (double2*)g_dev, a, b, mused);
}

int asr_chains_run(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz, int mode,
                   double depth_tol, int tail, int precision, int project, double* g, double* a, double* b, int* mused) {
  if (!ctx || !z || !g) { set_error("asr_chains_run: null argument"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  if (nz < 0 || ngroup < 1) { set_error("asr_chains_run: bad argument"); return ASR_EINVAL; }
  cudaStream_t s = ctx->stream;
  const size_t ng = (size_t)nz * ngroup;
  Dev<double2> d_z, d_g;   // freed on every return path
  ASR_TRY(d_z.alloc(nz));
  ASR_TRY(d_g.alloc(ng));
  ASR_CUDA(cudaMemcpyAsync(d_z.p, z, nz * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_TRY(chains_common(ctx, op, groups, ngroup, d_z.p, nz, mode, depth_tol, tail, precision, project, d_g.p, a, b, mused));
  ASR_CUDA(cudaMemcpyAsync(g, d_g.p, ng * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  return ASR_OK;
}

// dos_final (src/asr_class_scf.f90:1912-1931): uniform real energies, the chains of every group there, and the l-resolved
// sum -worb Im G / pi per (component, spin)
int asr_dos_final(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const int* comp, const int* spin,
                  const int* lorb, const double* worb, int ncomp, int nspin, double emin, double emax, double eta, int ndos,
                  double depth_tol, int tail, int precision, double* edos_e, double* edos) {
  if (!ctx || !op || !groups || ngroup < 1 || !comp || !spin || !lorb || !worb || ncomp < 1 || nspin < 1 || ndos < 1 ||
      !edos_e || !edos) {
    set_error("asr_dos_final: bad argument");
    return ASR_EINVAL;
  }
  for (int q = 0; q < ngroup; ++q) {
    if (comp[q] < 1 || comp[q] > ncomp || spin[q] < 1 || spin[q] > nspin || lorb[q] < 0 || lorb[q] > 2) {
      set_error("asr_dos_final: group %d has component, spin or l out of range", q + 1);
      return ASR_EINVAL;
    }
  }
  std::vector<double> z(2 * (size_t)ndos);
  for (int ie = 0; ie < ndos; ++ie) {
    edos_e[ie] = emin + (emax - emin) * ie / (double)std::max(ndos - 1, 1);
    z[2 * ie] = edos_e[ie];
    z[2 * ie + 1] = eta;
  }
  std::vector<double> g(2 * (size_t)ndos * ngroup);
  ASR_TRY(asr_chains_run(ctx, op, groups, ngroup, z.data(), ndos, ASR_MODE_EDC, depth_tol, tail, precision, 1, g.data(),
                         nullptr, nullptr, nullptr));
  std::fill(edos, edos + (size_t)ndos * 3 * ncomp * nspin, 0.0);
  const double pi = 3.14159265358979323846;
  for (int q = 0; q < ngroup; ++q) {
    double* out = edos + (size_t)ndos * (lorb[q] + 3 * ((comp[q] - 1) + (size_t)ncomp * (spin[q] - 1)));
    for (int ie = 0; ie < ndos; ++ie) out[ie] -= worb[q] * g[2 * ((size_t)ie + (size_t)ndos * q) + 1] / pi;
  }
  return ASR_OK;
}

// edc_green_proj (src/asr_edc.f90:174-232) for every (group, energy): all nlev steps (no depth test), g (nz, ngroup),
// gp / gp4 (9, nt, nz, ngroup) complex, mused (nz, ngroup) optional.  tnode, tgop (nsmax, nt) 1-based as returned by
// asr_op_build_targets; tw (9, nsmax, nt, ngroup) the dressing weights of every group.
int asr_chains_proj(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz, int tail,
                    int precision, int project, int nt, const int* tnode, const int* tgop, const double* tw, double* g,
                    double* gp, double* gp4, int* mused) {
  if (!ctx || !op || !groups || ngroup < 1 || !z || nz < 1 || nt < 1 || !tnode || !tgop || !tw || !g || !gp || !gp4) {
    set_error("asr_chains_proj: bad argument");
    return ASR_EINVAL;
  }
  if (tail < 0 || tail > 3) { set_error("asr_chains_proj: unknown tail"); return ASR_EINVAL; }
  const int nsm = op->nsmax;
  std::vector<int> tn((size_t)nsm * nt), tg((size_t)nsm * nt);
  for (size_t q = 0; q < tn.size(); ++q) {
    if (tnode[q] < 0 || tnode[q] > op->nn) { set_error("asr_chains_proj: target node out of range"); return ASR_EINVAL; }
    if (tnode[q] > 0 && (tgop[q] < 1 || tgop[q] > op->nop)) { set_error("asr_chains_proj: target operation out of range"); return ASR_EINVAL; }
    tn[q] = tnode[q] > 0 ? op->dev_node(tnode[q] - 1) : -1;   // reference numbering -> the device's node order
    tg[q] = tnode[q] > 0 ? tgop[q] - 1 : 0;
  }
  ASR_ON_DEVICE(ctx->device);
  cudaStream_t s = ctx->stream;
  GroupLayout GL = layout(op);
  std::vector<double> blob((size_t)GL.stride * ngroup, 0.0);
  std::vector<GroupInfo> gi(ngroup);
  for (int q = 0; q < ngroup; ++q) {
    const asr_chain_group& G = groups[q];
    if (!G.c || !G.d) { set_error("asr_chains_proj: group %d without c or d", q + 1); return ASR_EINVAL; }
    if (G.nlev < 1 || G.nlev > NLMAX) { set_error("asr_chains_proj: depth %d out of range 1..%d", G.nlev, NLMAX); return ASR_EINVAL; }
    ASR_TRY(make_group(op, GL, G.c, G.d, G.o, G.e, G.pa, G.pb, G.frozen_sp, G.start_orb, G.nlev, nullptr,
                       blob.data() + (size_t)GL.stride * q, gi[q]));
  }
  RunOptions opt;
  opt.mode = ASR_MODE_EDC;
  opt.depth_tol = 0.0;   // edc_green_proj runs every step
  opt.tail = tail;
  opt.precision = precision;
  opt.project = project;
  const int nlane = ngroup * nz;
  const size_t nout = (size_t)nlane * 9 * nt;
  std::vector<int> lg(nlane);
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nz; ++j) lg[(size_t)q * nz + j] = q;
  std::vector<double2> lz(nlane);
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nz; ++j) lz[(size_t)q * nz + j] = make_double2(z[2 * j], z[2 * j + 1]);
  Dev<double2> d_lz, d_g, d_gp, d_gp4;
  Dev<int> d_tn, d_tg;
  Dev<double> d_tw;
  ASR_TRY(d_lz.alloc(nlane)); ASR_TRY(d_g.alloc(nlane)); ASR_TRY(d_gp.alloc(nout)); ASR_TRY(d_gp4.alloc(nout));
  ASR_TRY(d_tn.alloc(tn.size())); ASR_TRY(d_tg.alloc(tg.size())); ASR_TRY(d_tw.alloc((size_t)9 * nsm * nt * ngroup));
  ASR_CUDA(cudaMemcpyAsync(d_lz.p, lz.data(), nlane * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_tn.p, tn.data(), tn.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_tg.p, tg.data(), tg.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_tw.p, tw, (size_t)9 * nsm * nt * ngroup * sizeof(double), cudaMemcpyHostToDevice, s));
  ProjSpec P;
  P.nt = nt; P.nsm = nsm; P.tnode = d_tn.p; P.tgop = d_tg.p; P.tw = d_tw.p; P.gp = d_gp.p; P.gp4 = d_gp4.p;
  std::vector<int> hm;
  int64_t nfall = 0, nsteps = 0;
  ASR_TRY(run_lanes(ctx, op, gi, blob, GL, lg, d_lz.p, nlane, opt, d_g.p, nullptr, nullptr, &hm, &nfall, &nsteps, &P));
  ASR_CUDA(cudaMemcpyAsync(g, d_g.p, nlane * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(gp, d_gp.p, nout * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(gp4, d_gp4.p, nout * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  if (mused) for (int L = 0; L < nlane; ++L) mused[L] = hm[L];
  ctx->nchain += nlane;
  ctx->nfall += nfall;
  return ASR_OK;
}

// Batch-shape autotuner: times (device time of the batches, best of two) the chains of the given groups (depth capped at
// `levels`, at most 64 of the energies) with
// 4, 8, 16, 32 tiles per batch at 4 nodes per warp, then 1, 2, 4, 8 nodes per warp at the best batch, and keeps the
// fastest pair on the operator for this precision (used whenever a call leaves the shape automatic).  times (8) receives
// the device times in ms (-1 where a candidate was skipped), or NULL.
int asr_autotune(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz, int precision,
                 int levels, int* tpb_out, int* npw_out, double* times) {
  if (!ctx || !op || !groups || ngroup < 1 || !z || nz < 1 || levels < 1) { set_error("asr_autotune: bad argument"); return ASR_EINVAL; }
  if (precision != ASR_FP64 && precision != ASR_FP32) { set_error("asr_autotune: unknown precision"); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  GroupLayout GL = layout(op);
  std::vector<double> blob((size_t)GL.stride * ngroup, 0.0);
  std::vector<GroupInfo> gi(ngroup);
  for (int q = 0; q < ngroup; ++q) {
    const asr_chain_group& G = groups[q];
    if (!G.c || !G.d) { set_error("asr_autotune: group %d without c or d", q + 1); return ASR_EINVAL; }
    int nl = std::min(std::max(G.nlev, 1), std::min(levels, NLMAX));
    ASR_TRY(make_group(op, GL, G.c, G.d, G.o, G.e, G.pa, G.pb, G.frozen_sp, G.start_orb, nl, nullptr,
                       blob.data() + (size_t)GL.stride * q, gi[q]));
  }
  const int nzt = std::min(nz, 64), nlane = ngroup * nzt;
  std::vector<int> lg(nlane);
  std::vector<double2> lz(nlane);
  for (int q = 0; q < ngroup; ++q)
    for (int j = 0; j < nzt; ++j) { lg[(size_t)q * nzt + j] = q; lz[(size_t)q * nzt + j] = make_double2(z[2 * j], z[2 * j + 1]); }
  Dev<double2> d_lz, d_g;
  ASR_TRY(d_lz.alloc(nlane)); ASR_TRY(d_g.alloc(nlane));
  ASR_CUDA(cudaMemcpy(d_lz.p, lz.data(), nlane * sizeof(double2), cudaMemcpyHostToDevice));
  const int ntile = ngroup * ((nzt + TL - 1) / TL);
  const int pix = precision == ASR_FP64 ? 0 : 1;
  auto timed = [&](int tpb, int npw, double& ms) -> int {
    RunOptions opt;
    opt.mode = ASR_MODE_EDC; opt.tail = ASR_TAIL_HULL; opt.precision = precision; opt.project = 1;
    opt.tiles_per_batch = tpb; opt.nodes_per_warp = npw;
    int64_t nf = 0, ns = 0;
    ms = 1e300;
    for (int rep = 0; rep < 2; ++rep) {   // device time of the batches (allocations excluded), best of two
      double t = 0.0;
      ASR_TRY(run_lanes(ctx, op, gi, blob, GL, lg, d_lz.p, nlane, opt, d_g.p, nullptr, nullptr, nullptr, &nf, &ns, nullptr, &t));
      ms = std::min(ms, t);
    }
    return ASR_OK;
  };
  // the tuned state is only replaced when every timing succeeded: a failed timing leaves the operator's previous (or
  // pinned) shape and link choice in place
  struct Restore {
    asr_op* op;
    int pix, tpb, npw, link;
    bool done = false;
    ~Restore() {
      if (!done) { op->tuned_tpb[pix] = tpb; op->tuned_npw[pix] = npw; op->tuned_link[pix] = link; }
    }
  } keep{op, pix, op->tuned_tpb[pix], op->tuned_npw[pix], op->tuned_link[pix]};
  op->tuned_link[pix] = 0;   // the shapes are timed with the general step kernel
  const int tpbs[4] = {4, 8, 16, 32}, npws[4] = {1, 2, 4, 8};
  double tab[8];
  for (double& t : tab) t = -1.0;
  double warm;
  ASR_TRY(timed(4, 4, warm));
  // a candidate replaces the built-in default (16 tiles in FP64, 8 in FP32, 4 nodes per warp) only when it is at least
  // 3 % faster: the timings carry a few per cent of noise, and the default is the measured best on the reference workload
  const int def_t = precision == ASR_FP64 ? 16 : 8, def_n = 4;
  const double margin = 0.97;
  for (int c = 0; c < 4; ++c) {
    if (tpbs[c] > ntile && tpbs[c] != def_t) continue;
    ASR_TRY(timed(tpbs[c], def_n, tab[c]));
  }
  int best_t = def_t, best_n = def_n;
  double best = tab[def_t == 16 ? 2 : 1];
  for (int c = 0; c < 4; ++c)
    if (tab[c] > 0 && tab[c] < margin * best) { best = tab[c]; best_t = tpbs[c]; }
  for (int c = 0; c < 4; ++c) ASR_TRY(timed(best_t, npws[c], tab[4 + c]));
  best = tab[4 + 2];   // 4 nodes per warp
  for (int c = 0; c < 4; ++c)
    if (tab[4 + c] < margin * best) { best = tab[4 + c]; best_n = npws[c]; }
  op->tuned_tpb[pix] = best_t;
  op->tuned_npw[pix] = best_n;
  // then the step kernel with fixed-offset link gathers at that shape (the same bits; kept when it is 3 % faster)
  double t_gen = 0.0, t_link = 0.0;
  ASR_TRY(timed(best_t, best_n, t_gen));
  op->tuned_link[pix] = 1;
  int rc = timed(best_t, best_n, t_link);
  if (rc != ASR_OK) return rc;
  op->tuned_link[pix] = t_link < margin * t_gen ? 1 : 0;
  keep.done = true;
  op->tuned_link_ms[pix][0] = t_gen;
  op->tuned_link_ms[pix][1] = t_link;
  if (tpb_out) *tpb_out = best_t;
  if (npw_out) *npw_out = best_n;
  if (times) for (int c = 0; c < 8; ++c) times[c] = tab[c];
  return ASR_OK;
}

int asr_op_tuning(const asr_op* op, int precision, int* tpb, int* npw, int* link, double* ms) {
  if (!op || (precision != ASR_FP64 && precision != ASR_FP32)) { set_error("asr_op_tuning: bad argument"); return ASR_EINVAL; }
  const int pix = precision == ASR_FP64 ? 0 : 1;
  if (tpb) *tpb = op->tuned_tpb[pix];
  if (npw) *npw = op->tuned_npw[pix];
  if (link) *link = op->tuned_link[pix];
  if (ms) { ms[0] = op->tuned_link_ms[pix][0]; ms[1] = op->tuned_link_ms[pix][1]; }
  return ASR_OK;
}

int asr_op_set_tuning(asr_op* op, int precision, int tpb, int npw, int link) {
  if (!op || (precision != ASR_FP64 && precision != ASR_FP32)) { set_error("asr_op_set_tuning: bad argument"); return ASR_EINVAL; }
  if (!(tpb == 0 || tpb == 4 || tpb == 8 || tpb == 16 || tpb == 32)) { set_error("asr_op_set_tuning: tiles per batch %d", tpb); return ASR_EINVAL; }
  if (!(npw == 0 || npw == 1 || npw == 2 || npw == 4 || npw == 8)) { set_error("asr_op_set_tuning: nodes per warp %d", npw); return ASR_EINVAL; }
  if (link != 0 && link != 1) { set_error("asr_op_set_tuning: link must be 0 or 1"); return ASR_EINVAL; }
  const int pix = precision == ASR_FP64 ? 0 : 1;
  op->tuned_tpb[pix] = tpb;
  op->tuned_npw[pix] = npw;
  op->tuned_link[pix] = link;
  return ASR_OK;
}

int asr_cf_eval(asr_ctx* ctx, const double* a, const double* b, const int* m, int ld, int nchain, const double* z, int nz, int tail,
                double* g, double* edges, int64_t* nfall) {
  if (!ctx || !a || !b || !m || !z || !g || ld < 1 || nchain < 1 || nz < 1) { set_error("asr_cf_eval: bad argument"); return ASR_EINVAL; }
  for (int c = 0; c < nchain; ++c)
    if (m[c] < 1 || m[c] > ld || m[c] > CF_NMAX) { set_error("asr_cf_eval: depth of chain %d out of range", c + 1); return ASR_EINVAL; }
  ASR_ON_DEVICE(ctx->device);
  cudaStream_t s = ctx->stream;
  size_t nab = (size_t)ld * nchain, nzz = (size_t)nz * nchain;
  Dev<double2> d_a, d_b, d_z, d_g, d_e;   // freed on every return path
  Dev<int> d_m, d_nf;
  ASR_TRY(d_a.alloc(nab)); ASR_TRY(d_b.alloc(nab)); ASR_TRY(d_z.alloc(nzz)); ASR_TRY(d_g.alloc(nzz));
  ASR_TRY(d_m.alloc(nchain)); ASR_TRY(d_nf.alloc(1));
  if (edges) ASR_TRY(d_e.alloc(2 * nzz));
  ASR_CUDA(cudaMemcpyAsync(d_a.p, a, nab * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_b.p, b, nab * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_z.p, z, nzz * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_m.p, m, nchain * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemsetAsync(d_nf.p, 0, sizeof(int), s));
  k_cf_eval<<<(unsigned)((nzz + 127) / 128), 128, 0, s>>>(d_a.p, d_b.p, d_m.p, ld, nchain, d_z.p, nz, tail, d_g.p,
                                                          edges ? d_e.p : nullptr, d_nf.p);
  int nf = 0;
  ASR_CUDA(cudaGetLastError());
  ctx->launches += 1;
  ASR_CUDA(cudaMemcpyAsync(g, d_g.p, nzz * sizeof(double2), cudaMemcpyDeviceToHost, s));
  if (edges) ASR_CUDA(cudaMemcpyAsync(edges, d_e.p, 2 * nzz * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(&nf, d_nf.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  if (nfall) *nfall = nf;
  ctx->nfall += nf;
  return ASR_OK;
}

// reverse mode of one terminated fraction (host): abar/bbar(m) complex receive w dG/da_k, w dG/db_k
int asr_cf_adjoint(const double* a, const double* b, int m, double zr, double zi, int tail, double wr, double wi, double* abar,
                   double* bbar, double* g) {
  if (!a || !b || !abar || !bbar || m < 1 || m > CF_NMAX || tail < 0 || tail > 3) {
    set_error("asr_cf_adjoint: bad argument (tails none, hull, bp, avg2; 1 <= m <= %d)", CF_NMAX);
    return ASR_EINVAL;
  }
  std::vector<double2> gt(m), v(m), t(m), wd(m), we(m);
  for (int k = 0; k < m; ++k) { ((double2*)abar)[k] = make_double2(0, 0); ((double2*)bbar)[k] = make_double2(0, 0); }
  double2 G = cf_species_adjoint((const double2*)a, (const double2*)b, m, make_double2(zr, zi), tail, make_double2(wr, wi),
                                 (double2*)abar, (double2*)bbar, gt.data(), v.data(), t.data(), wd.data(), we.data());
  if (g) { g[0] = G.x; g[1] = G.y; }
  return ASR_OK;
}

// ---- contour (src/asr_contour.f90), host
static const double PI_ = 3.14159265358979323846264338327950288;

int asr_gauss_legendre(int n, double* x, double* w) {   // :132-151
  if (n < 1 || !x || !w) { set_error("gauss_legendre: bad argument"); return ASR_EINVAL; }
  for (int i = 1; i <= (n + 1) / 2; ++i) {
    double z = std::cos(PI_ * (i - 0.25) / (n + 0.5)), z1, p1 = 1, p2 = 0, p3, pp = 1;
    for (int it = 0; it < 100; ++it) {
      p1 = 1.0; p2 = 0.0;
      for (int k = 1; k <= n; ++k) { p3 = p2; p2 = p1; p1 = ((2 * k - 1) * z * p2 - (k - 1) * p3) / k; }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1.0e-15) break;
    }
    x[i - 1] = -z; x[n - i] = z;
    w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp); w[n - i] = w[i - 1];
  }
  return ASR_OK;
}

static void put_node(double* z, double* w, int k, double zr, double zi, double wr, double wi) {
  z[2 * k] = zr; z[2 * k + 1] = zi; w[2 * k] = wr; w[2 * k + 1] = wi;
}

int asr_contour_nodes(double ebot, double ef, int n, double eta_end, double* z, double* w) {   // :17-34
  if (n < 1 || !z || !w || !(ef > ebot)) { set_error("contour_nodes: bad argument"); return ASR_EINVAL; }
  std::vector<double> x(n), wg(n);
  asr_gauss_legendre(n, x.data(), wg.data());
  double c = 0.5 * (ebot + ef), r = 0.5 * (ef - ebot), th0 = 0.0;
  if (eta_end >= 0.0) th0 = std::asin(std::min(eta_end / r, 0.5));
  for (int j = 0; j < n; ++j) {
    double th = th0 + 0.5 * (PI_ - th0) * (1.0 - x[j]);
    double f = wg[j] * (-0.5 * (PI_ - th0));
    // w = f * (i r) * exp(i th) = f r (-sin th + i cos th)
    put_node(z, w, j, c + r * std::cos(th), r * std::sin(th), -f * r * std::sin(th), f * r * std::cos(th));
  }
  return ASR_OK;
}

int asr_contour_nodes_closed(double ebot, double ef, double eta, int na, int nv, double* z, double* w) {   // :39-58
  if (na < 1 || nv < 1 || !z || !w || !(ef > ebot) || !(eta > 0)) { set_error("contour_nodes_closed: bad argument"); return ASR_EINVAL; }
  std::vector<double> xa(na), wa(na), xv(nv), wv(nv);
  asr_gauss_legendre(na, xa.data(), wa.data());
  asr_gauss_legendre(nv, xv.data(), wv.data());
  double c = (ef * ef + eta * eta - ebot * ebot) / (2.0 * (ef - ebot)), r = c - ebot, th0 = std::atan2(eta, ef - c);
  for (int j = 0; j < na; ++j) {
    double th = th0 + 0.5 * (PI_ - th0) * (1.0 - xa[j]);
    double f = wa[j] * (-0.5 * (PI_ - th0));
    put_node(z, w, j, c + r * std::cos(th), r * std::sin(th), -f * r * std::sin(th), f * r * std::cos(th));
  }
  for (int j = 0; j < nv; ++j) put_node(z, w, na + j, ef, 0.5 * eta * (1.0 + xv[j]), 0.0, -0.5 * eta * wv[j]);
  return ASR_OK;
}

int asr_contour_nodes_fermi(double ebot, double mu, double kt, int npole, int nmain, int nstep, double* z, double* w) {   // :77-121
  if (!z || !w || kt <= 0.0 || npole < 0 || nmain < 1 || nstep < 1) { set_error("contour_nodes_fermi: bad argument"); return ASR_EINVAL; }
  auto fermi_r = [&](double e) { double t = (e - mu) / kt; return t > 0.0 ? std::exp(-t) / (1.0 + std::exp(-t)) : 1.0 / (1.0 + std::exp(t)); };
  double gam = 2.0 * npole * PI_ * kt;
  std::vector<double> xv(4), wv(4), xm(nmain), wm(nmain), xs(nstep), ws(nstep), xt(8), wt(8);
  asr_gauss_legendre(4, xv.data(), wv.data()); asr_gauss_legendre(nmain, xm.data(), wm.data());
  asr_gauss_legendre(nstep, xs.data(), ws.data()); asr_gauss_legendre(8, xt.data(), wt.data());
  int k = 0;
  for (int j = 0; j < 4; ++j) {   // vertical leg at E_bot: complex Fermi factor
    double zr = ebot, zi = 0.5 * gam * (1.0 + xv[j]);
    double tr = (zr - mu) / kt, ti = zi / kt;
    double fr = 1.0, fi = 0.0;
    if (tr >= -600.0) {   // 1 / (exp(t) + 1)
      double er = std::exp(tr) * std::cos(ti) + 1.0, ei = std::exp(tr) * std::sin(ti), den = er * er + ei * ei;
      fr = er / den; fi = -ei / den;
    }
    double wr = -0.5 * gam * wv[j] * fi, wi = 0.5 * gam * wv[j] * fr;   // (i g) * f
    put_node(z, w, k++, zr, zi, wr, wi);
  }
  double lo = ebot, hi = mu - 10.0 * kt;
  for (int j = 0; j < nmain; ++j) { double x = 0.5 * (lo + hi) + 0.5 * (hi - lo) * xm[j]; put_node(z, w, k++, x, gam, 0.5 * (hi - lo) * wm[j] * fermi_r(x), 0.0); }
  lo = mu - 10.0 * kt; hi = mu + 10.0 * kt;
  for (int j = 0; j < nstep; ++j) { double x = 0.5 * (lo + hi) + 0.5 * (hi - lo) * xs[j]; put_node(z, w, k++, x, gam, 0.5 * (hi - lo) * ws[j] * fermi_r(x), 0.0); }
  lo = mu + 10.0 * kt; hi = mu + 40.0 * kt;
  for (int j = 0; j < 8; ++j) { double x = 0.5 * (lo + hi) + 0.5 * (hi - lo) * xt[j]; put_node(z, w, k++, x, gam, 0.5 * (hi - lo) * wt[j] * fermi_r(x), 0.0); }
  for (int j = 0; j < npole; ++j) put_node(z, w, k++, mu, (2 * j + 1) * PI_ * kt, 0.0, -2.0 * PI_ * kt);
  return ASR_OK;
}

int asr_contour_moment(const double* z, const double* w, const double* g, int n, double enu, int k, double* m) {   // :124-130
  if (!z || !w || !g || !m || n < 0 || k < 0) { set_error("contour_moment: bad argument"); return ASR_EINVAL; }
  double sr = 0.0, si = 0.0;
  for (int j = 0; j < n; ++j) {
    double pr = 1.0, pim = 0.0, xr = z[2 * j] - enu, xi = z[2 * j + 1];
    for (int q = 0; q < k; ++q) { double t = pr * xr - pim * xi; pim = pr * xi + pim * xr; pr = t; }
    double ar = w[2 * j] * pr - w[2 * j + 1] * pim, ai = w[2 * j] * pim + w[2 * j + 1] * pr;
    sr += ar * g[2 * j] - ai * g[2 * j + 1];
    si += ar * g[2 * j + 1] + ai * g[2 * j];
  }
  *m = -si / PI_;
  return ASR_OK;
}

}  // extern "C"
