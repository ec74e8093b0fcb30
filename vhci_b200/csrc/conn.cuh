// Device helpers shared by the Hamiltonian and PT2 kernels: connection-group targets and the
// FC term sums that give Hamiltonian elements.
#pragma once

#include "ops.h"

namespace vhci {

// Sum of a group's terms for ket key k: each term is fc * prod_j T[pw_j][q(mode_j)][dl_j], multiplied
// left to right and summed in table order (the reference's AnharmPot product and Vij sum order).
// Products and sums use explicit round-to-nearest operations so no multiply-add is contracted:
// the results are the same bits as the reference's separate multiplies and adds.
template <int W>
__device__ __forceinline__ double group_value(const ConnDev& cd, int tb, int te,
                                              const uint64_t (&k)[W], const KeyLayout& L) {
  const int qs = L.qmax + 1;
  double v = 0.0;
  for (int t = tb; t < te; ++t) {
    const TermDev tm = cd.terms[t];
    double tv = tm.fc;
    for (int j = 0; j < tm.nk; ++j) {
      const int q = key_q<W>(k, tm.mode[j], L.mpw, L.bits);
      tv = __dmul_rn(tv, __ldg(cd.T + ((int64_t)tm.pw[j] * qs + q) * 13 + tm.dl[j] + 6));
    }
    v = __dadd_rn(v, tv);
  }
  return v;
}

// Diagonal element: harmonic energy (Ham.cpp:211-220 operation order) plus the Delta = 0 terms
// in table order (quartic then sextic); equals the reference's fl(E_i + V_ii).
template <int W>
__device__ __forceinline__ double diag_value(const ConnDev& cd, const uint64_t (&k)[W],
                                             const KeyLayout& L) {
  double e = 0.0;
  for (int m = 0; m < cd.nm; ++m) {
    double ej = 0.5;
    ej = __dadd_rn(ej, (double)key_q<W>(k, m, L.mpw, L.bits));
    ej = __dmul_rn(ej, __ldg(cd.freq + m));
    e = __dadd_rn(e, ej);
  }
  const int qs = L.qmax + 1;
  double v = 0.0;
  for (int t = 0; t < cd.ndterms; ++t) {
    const TermDev tm = cd.dterms[t];
    double tv = tm.fc;
    for (int j = 0; j < tm.nk; ++j) {
      const int q = key_q<W>(k, tm.mode[j], L.mpw, L.bits);
      tv = __dmul_rn(tv, __ldg(cd.T + ((int64_t)tm.pw[j] * qs + q) * 13 + 6));
    }
    v = __dadd_rn(v, tv);
  }
  return __dadd_rn(e, v);
}

// Target of group u from key k, or false when a changed mode leaves [0, qmax] (such a state
// cannot be in a basis stored with this layout).
template <int W>
__device__ __forceinline__ bool group_target(const ConnDev& cd, int64_t u, const GroupDev& g,
                                             const uint64_t (&k)[W], const KeyLayout& L,
                                             uint64_t (&t)[W]) {
  for (int c = 0; c < g.nchg; ++c) {
    const int q = key_q<W>(k, g.mode[c], L.mpw, L.bits) + g.delta[c];
    if (q < 0 || q > L.qmax) return false;
  }
#pragma unroll
  for (int w = 0; w < W; ++w) t[w] = k[w] + (uint64_t)__ldg(cd.wdelta + u * W + w);
  return true;
}

}  // namespace vhci
