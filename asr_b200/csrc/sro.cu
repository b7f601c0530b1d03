// Species layouts with first-shell short-range order for the explicit-supercell (KPM) workloads.
//
// The reference generates such layouts with a Python SQS tool and a C Monte Carlo helper (tools/sqs.py, tools/
// sro_closure/sro_mc.c); this is an independent implementation: species swap moves on the site lattice, accepted by the
// Metropolis rule on the objective F = sum_{a <= b} (N_ab - N*_ab)^2, where N_ab counts first-shell (site, neighbour)
// pairs of species (a, b) and N*_ab = n z x_a x_b (1 - alpha_ab) is the count of the target Warren-Cowley parameters
// alpha_ab (unlike pairs given, like pairs implied by sum_b x_b alpha_ab = 0).  The temperature falls geometrically;
// the counter-based generator makes the layout a function of the seed alone.  Host code.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/asr_b200.h"
#include "common.cuh"

namespace {

struct Rng {   // splitmix64 stream
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  uint64_t below(uint64_t n) { return next() % n; }
};

}  // namespace

extern "C" int asr_sro_layout(int nsite, int z, const int* nbr, int ldnbr, int nsp, const double* conc, const double* alpha,
                              uint64_t seed, int sweeps, int* spc, double* alpha_out) {
  if (nsite < 2 || z < 1 || z > ldnbr || !nbr || nsp < 1 || nsp > 16 || !conc || !spc) {
    asrb::set_error("asr_sro_layout: bad argument");
    return ASR_EINVAL;
  }
  Rng rng{seed * 0x9E3779B97F4A7C15ULL + 12345};
  // exact composition, seeded shuffle
  std::vector<int> s(nsite);
  {
    int k = 0;
    double acc = 0.0;
    for (int a = 0; a < nsp; ++a) {
      acc += conc[a];
      int upto = (a == nsp - 1) ? nsite : (int)std::llround(acc * nsite);
      for (; k < upto && k < nsite; ++k) s[k] = a;
    }
    for (int i = nsite - 1; i > 0; --i) std::swap(s[i], s[rng.below(i + 1)]);
  }
  std::vector<double> x(nsp, 0.0);
  for (int i = 0; i < nsite; ++i) x[s[i]] += 1.0;
  for (int a = 0; a < nsp; ++a) x[a] /= nsite;
  // target counts (ordered pairs: every site with each of its z first-shell neighbours)
  std::vector<double> al((size_t)nsp * nsp, 0.0), tgt((size_t)nsp * nsp);
  if (alpha)
    for (int a = 0; a < nsp; ++a)
      for (int b = 0; b < nsp; ++b) if (a != b) al[a * nsp + b] = alpha[a + (size_t)nsp * b];
  for (int a = 0; a < nsp; ++a) {
    double sum = 0.0;
    for (int b = 0; b < nsp; ++b) if (b != a) sum += x[b] * al[a * nsp + b];
    al[a * nsp + a] = x[a] > 0 ? -sum / x[a] : 0.0;
  }
  for (int a = 0; a < nsp; ++a)
    for (int b = 0; b < nsp; ++b) tgt[a * nsp + b] = (double)nsite * z * x[a] * x[b] * (1.0 - al[a * nsp + b]);
  std::vector<double> N((size_t)nsp * nsp, 0.0);
  for (int i = 0; i < nsite; ++i)
    for (int k = 0; k < z; ++k) N[s[i] * nsp + s[nbr[k + (size_t)ldnbr * i] - 1]] += 1.0;
  auto F = [&](const std::vector<double>& M) {
    double f = 0.0;
    for (int q = 0; q < nsp * nsp; ++q) f += (M[q] - tgt[q]) * (M[q] - tgt[q]);
    return f;
  };
  double f = F(N);
  std::vector<double> dN((size_t)nsp * nsp);
  const long nprop = (long)std::max(sweeps, 1) * nsite;
  double T = f / (double)nsite + 1.0;
  const double Tend = 1e-3;
  const double cool = std::pow(Tend / T, 1.0 / (double)nprop);
  for (long it = 0; it < nprop; ++it, T *= cool) {
    int i = (int)rng.below(nsite), j = (int)rng.below(nsite);
    int a = s[i], b = s[j];
    if (a == b) continue;
    std::fill(dN.begin(), dN.end(), 0.0);
    // pairs touching i or j, counted in both directions; a pair (i, j) itself is handled by swapping on a copy
    auto sub_site = [&](int p, double w) {
      int sp = s[p];
      for (int k = 0; k < z; ++k) {
        int q = nbr[k + (size_t)ldnbr * p] - 1;
        int sq = s[q];
        dN[sp * nsp + sq] += w;
        dN[sq * nsp + sp] += w;
      }
    };
    // remove the old pairs of i and j (a pair i-j is removed twice: add it back once)
    sub_site(i, -1.0);
    sub_site(j, -1.0);
    int nij = 0;
    for (int k = 0; k < z; ++k) if (nbr[k + (size_t)ldnbr * i] - 1 == j) ++nij;
    if (nij) { dN[a * nsp + b] += nij; dN[b * nsp + a] += nij; }
    std::swap(s[i], s[j]);
    sub_site(i, +1.0);
    sub_site(j, +1.0);
    if (nij) { dN[b * nsp + a] -= nij; dN[a * nsp + b] -= nij; }
    for (int q = 0; q < nsp * nsp; ++q) dN[q] += N[q];
    double fn = F(dN);
    if (fn <= f || rng.uniform() < std::exp(-(fn - f) / T)) {
      N.swap(dN);
      f = fn;
    } else {
      std::swap(s[i], s[j]);
    }
  }
  for (int i = 0; i < nsite; ++i) spc[i] = s[i] + 1;
  if (alpha_out)
    for (int a = 0; a < nsp; ++a)
      for (int b = 0; b < nsp; ++b) {
        double p = N[a * nsp + b] / ((double)nsite * z * x[a]);   // P(b | a) in the first shell
        alpha_out[a + (size_t)nsp * b] = x[b] > 0 ? 1.0 - p / x[b] : 0.0;
      }
  return ASR_OK;
}
