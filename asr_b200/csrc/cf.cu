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
