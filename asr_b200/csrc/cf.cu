// Continued-fraction kernels: many (chain, energy) fractions with the reference's tails (cf_species,
// src/asr_chain.f90:67-167) and the real-chain terminators of the plain route (make_terminator / terminated_green,
// src/reference/asr_terminator.f90:83-126).
#include "cf.cuh"
#include "op.h"

namespace asrb {

// g(j, c) = cf_species(a(:, c), b(:, c), m(c), z(j, c), tail); one thread per (energy, chain)
__global__ void k_cf_eval(const double2* a, const double2* b, const int* m, int ld, int nchain, const double2* z, int nz, int tail,
                          double2* g, double2* edges, int* nfall) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nz * nchain) return;
  int c = (int)(t / nz);
  int mc = m[c];
  if (mc < 1 || mc > CF_NMAX) { g[t] = make_double2(0.0, 0.0); return; }
  double2 wd[CF_NMAX], we[CF_NMAX];
  int nf = 0;
  double2 e2[2];
  g[t] = cf_species_dev(a + (size_t)ld * c, b + (size_t)ld * c, mc, z[t], tail, wd, we, &nf, e2);
  if (edges) { edges[2 * t] = e2[0]; edges[2 * t + 1] = e2[1]; }
  if (nf) atomicAdd(nfall, nf);
}

// real chains: (ainf, binf) per chain for the plain route.  method: ASR_TAIL_BP beer-pettifor, ASR_TAIL_AVG2
// sqrt-avg2, ASR_TAIL_NONE no tail.
__global__ void k_real_tail(const double* a, const double* b, const int* n, int ld, int nchain, int method, double* ainf,
                            double* binf) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchain) return;
  const double* ac = a + (size_t)ld * c;
  const double* bc = b + (size_t)ld * c;
  int nc = n[c];
  double A = 0.0, B = 0.0;
  if (nc >= 2 && method == ASR_TAIL_BP) {
    double wd[CF_NMAX];
    bp_asymptote_dev(ac, bc, nc, wd, A, B);
  } else if (nc >= 2 && method == ASR_TAIL_AVG2) {
    A = 0.5 * (ac[nc - 1] + ac[nc - 2]);
    B = sqrt(0.5 * (bc[nc - 1] * bc[nc - 1] + bc[nc - 2] * bc[nc - 2]));
  }
  ainf[c] = A;
  binf[c] = B;
}

__global__ void k_real_green(const double* a, const double* b, const int* n, int ld, int nchain, const double* ainf,
                             const double* binf, int method, const double2* z, int nz, double2* g) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nz * nchain) return;
  int c = (int)(t / nz);
  int nc = n[c];
  if (nc < 1) { g[t] = make_double2(0, 0); return; }
  bool tail = method != ASR_TAIL_NONE && nc >= 2 && binf[c] != 0.0;
  g[t] = terminated_green_dev(a + (size_t)ld * c, b + (size_t)ld * c, nc, z[t % nz], ainf[c], binf[c], tail);
}

}  // namespace asrb

// ------------------------------------------------------------------------------------------------ asr_cf_eval_noalloc
// The same fractions as asr_cf_eval, staged through one file-scope device array instead of cudaMalloc'd buffers.  It is
// meant for callers that may not allocate device memory: a host that evaluates fractions between chain batches while
// other streams are busy (cudaMalloc and cudaFree synchronise the device), or a process whose device memory is owned by
// another allocator (a framework's caching allocator, a fixed memory budget).  The operands must fit in the scratch:
//   32 ld nchain (a, b) + 32 nz nchain (z, g) + 4 nchain (m) + 4 (fallback counter) bytes, each part rounded up to
//   256 bytes, at most ASR_CF_NOALLOC_BYTES (8 MiB) per device.
// Only the fallback counter has to start at zero; it is cleared on the stream before every launch.  The scratch is one
// per device: two calls that overlap in time on the same device (other host threads, other streams) race on it.
#include <mutex>

#include "../../include/asr_b200.h"

namespace asrb {
namespace {

__device__ __align__(256) unsigned char g_cf_scratch[ASR_CF_NOALLOC_BYTES];
std::mutex g_cf_mu;

size_t up256(size_t n) { return (n + 255) & ~(size_t)255; }

// device address of the scratch on the context's device, resolved on the first call with that device current and kept
// with the context (a context, like every device address it holds, does not outlive a reset of its device)
int cf_scratch(asr_ctx* ctx, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_cf_mu);
  if (!ctx->cf_scratch) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_cf_scratch);
    if (rc != cudaSuccess || !p) {
      set_error("asr_cf_eval_noalloc: cudaGetSymbolAddress failed on device %d: %s", ctx->device, cudaGetErrorString(rc));
      return ASR_ECUDA;
    }
    ctx->cf_scratch = (unsigned char*)p;
  }
  *out = ctx->cf_scratch;
  return ASR_OK;
}

}  // namespace
}  // namespace asrb

extern "C" int asr_cf_eval_noalloc(asr_ctx* ctx, const double* a, const double* b, const int* m, int ld, int nchain,
                                   const double* z, int nz, int tail, double* g, int64_t* nfall) {
  using namespace asrb;
  if (!ctx || !a || !b || !m || !z || !g || ld < 1 || nchain < 1 || nz < 1 || tail < 0 || tail > 3) {
    set_error("asr_cf_eval_noalloc: bad argument");
    return ASR_EINVAL;
  }
  for (int c = 0; c < nchain; ++c)
    if (m[c] < 1 || m[c] > ld || m[c] > CF_NMAX) { set_error("asr_cf_eval_noalloc: depth of chain %d out of range", c + 1); return ASR_EINVAL; }
  const size_t nab = (size_t)ld * nchain, nzz = (size_t)nz * nchain;
  const size_t o_b = up256(nab * sizeof(double2)), o_z = o_b + up256(nab * sizeof(double2));
  const size_t o_g = o_z + up256(nzz * sizeof(double2)), o_m = o_g + up256(nzz * sizeof(double2));
  const size_t o_nf = o_m + up256((size_t)nchain * sizeof(int)), total = o_nf + up256(sizeof(int));
  if (total > (size_t)ASR_CF_NOALLOC_BYTES) {
    set_error("asr_cf_eval_noalloc: the operands need %zu bytes, above the %zu-byte static scratch (split the chains)", total,
              (size_t)ASR_CF_NOALLOC_BYTES);
    return ASR_EINVAL;
  }
  ASR_ON_DEVICE(ctx->device);
  unsigned char* base = nullptr;
  ASR_TRY(cf_scratch(ctx, &base));
  cudaStream_t s = ctx->stream;
  double2* d_a = (double2*)base;
  double2* d_b = (double2*)(base + o_b);
  double2* d_z = (double2*)(base + o_z);
  double2* d_g = (double2*)(base + o_g);
  int* d_m = (int*)(base + o_m);
  int* d_nf = (int*)(base + o_nf);
  ASR_CUDA(cudaMemcpyAsync(d_a, a, nab * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_b, b, nab * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_z, z, nzz * sizeof(double2), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemcpyAsync(d_m, m, nchain * sizeof(int), cudaMemcpyHostToDevice, s));
  ASR_CUDA(cudaMemsetAsync(d_nf, 0, sizeof(int), s));
  k_cf_eval<<<(unsigned)((nzz + 127) / 128), 128, 0, s>>>(d_a, d_b, d_m, ld, nchain, d_z, nz, tail, d_g, nullptr, d_nf);
  ASR_CUDA(cudaGetLastError());
  ctx->launches += 1;
  int nf = 0;
  ASR_CUDA(cudaMemcpyAsync(g, d_g, nzz * sizeof(double2), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaMemcpyAsync(&nf, d_nf, sizeof(int), cudaMemcpyDeviceToHost, s));
  ASR_CUDA(cudaStreamSynchronize(s));
  if (nfall) *nfall = nf;
  ctx->nfall += nf;
  return ASR_OK;
}
