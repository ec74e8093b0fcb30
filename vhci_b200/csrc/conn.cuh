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

// ---- lowered-mode index: visit only the groups a state can move by --------------------------

// Binomial coefficients C(a, r) for a <= 32, r <= 6 at [a * kBinomR + r]; each block fills its
// shared copy once with fill_binom (followed by __syncthreads).
constexpr int kBinomA = 33, kBinomR = 7, kBinomElems = kBinomA * kBinomR;

__device__ __forceinline__ void fill_binom(uint32_t* binom) {
  for (int t = threadIdx.x; t < kBinomElems; t += blockDim.x) {
    const int a = t / kBinomR, r = t % kBinomR;
    uint64_t v = 1;  // C(a, i) after step i; exact at every step
    for (int i = 0; i < r; ++i) v = v * (uint64_t)(a > i ? a - i : 0) / (uint64_t)(i + 1);
    binom[t] = (uint32_t)v;
  }
}

// Segment of the groups lowering the mode set `key` (lowered_key layout): first group, count.
__device__ __forceinline__ void seg_find(const ConnDev& cd, uint64_t key, int& first, int& count) {
  uint32_t h = (uint32_t)mix64(key) & cd.lmask;
  for (uint32_t probe = 0; probe <= cd.lmask; ++probe) {  // load <= 1/2: ends at an empty slot
    const uint64_t k = __ldg(cd.lkey + h);
    if (k == key) {
      first = __ldg(cd.lseg + 2 * h);
      count = __ldg(cd.lseg + 2 * h + 1);
      return;
    }
    if (k == 0) return;
    h = (h + 1) & cd.lmask;
  }
}

// Calls body(u) for the connection groups u that state k can move by, in warp-uniform rounds:
// every lane runs body each round, with u = -1 on lanes that have no group that round.  A group
// lowering a mode that is not excited in k cannot apply, so with the index only the segments of
// the subsets of k's excited modes (sizes 0..maxl, r-major then colexicographic order) are
// visited; lanes share the flattened list of the found segments.  Without the index, or when the
// subsets outnumber half the groups, every group is visited.  The sequence depends on k alone,
// so count and fill passes see the same order.  `exc` is this warp's 128-byte scratch.
template <int W, class Body>
__device__ __forceinline__ void for_each_group(const ConnDev& cd, const uint64_t (&k)[W],
                                               const KeyLayout& L, uint8_t* exc,
                                               const uint32_t* binom, Body&& body) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int e = 0;
  int64_t nsub = -1;
  __syncwarp();  // the previous state's readers of exc are done
  if (cd.maxl >= 0) {
    for (int m0 = 0; m0 < cd.nm; m0 += 32) {
      const int m = m0 + lane;
      const bool x = m < cd.nm && key_q<W>(k, m, L.mpw, L.bits) > 0;
      const unsigned b = __ballot_sync(full, x);
      if (x) exc[e + __popc(b & lanemask_lt())] = (uint8_t)m;
      e += __popc(b);
    }
    __syncwarp();
    if (e < kBinomA) {
      nsub = 0;
      for (int r = 0; r <= cd.maxl && r <= e; ++r) nsub += binom[e * kBinomR + r];
      if (nsub > cd.ngroups / 2) nsub = -1;
    }
  }
  if (nsub < 0) {
    for (int64_t u0 = 0; u0 < cd.ngroups; u0 += 32)
      body(u0 + lane < cd.ngroups ? u0 + lane : (int64_t)-1);
    return;
  }
  for (int64_t s0 = 0; s0 < nsub; s0 += 32) {
    const int64_t s = s0 + lane;
    int first = 0, cnt = 0;
    if (s < nsub) {
      int r = 0;
      int64_t rem = s;
      while (rem >= (int64_t)binom[e * kBinomR + r]) rem -= binom[e * kBinomR + r++];
      uint64_t key = (uint64_t)(r + 1);
      int hi = e;  // element i = largest c < hi with C(c, i) <= rem (combinatorial number system)
      for (int i = r; i >= 1; --i) {
        int c = hi - 1;
        while ((int64_t)binom[c * kBinomR + i] > rem) --c;
        rem -= binom[c * kBinomR + i];
        key |= (uint64_t)(exc[c] + 1) << (3 + 7 * (i - 1));
        hi = c;
      }
      seg_find(cd, key, first, cnt);
    }
    int incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(full, incl, d);
      if (lane >= d) incl += v;
    }
    const int excl = incl - cnt;
    const int total = __shfl_sync(full, incl, 31);
    for (int f0 = 0; f0 < total; f0 += 32) {
      const int f = f0 + lane;
      int lo = 0;  // owner lane: the smallest j with incl_j > f
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1)
        if (__shfl_sync(full, incl, lo + step - 1) <= f) lo += step;
      const int j = lo < 32 ? lo : 31;
      const int ej = __shfl_sync(full, excl, j);
      const int fj = __shfl_sync(full, first, j);
      body(f < total ? (int64_t)(fj + f - ej) : (int64_t)-1);
    }
  }
}

}  // namespace vhci
