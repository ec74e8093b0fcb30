// Epstein-Nesbet PT2 kernels (reference: DoPT2, PT2.cpp:16-154).
//
// The reference loops over every (perturber a, variational state i) pair.  Here the connected
// pairs are generated from the variational side: for each state i and connection group u, the
// target a = i + Delta_u is looked up in the perturber hash; hits become entries (a, i, H_ai) of a
// perturber-row CSR (count pass, scan, fill pass).  A fused kernel then forms
// num_a[n] = sum_i H_ai C_in, E_a = H_aa, and sum_a num_a[n]^2 / (E_n - E_a) per block.
#include "conn.cuh"
#include "ops.h"

namespace vhci {

namespace {

inline int grid_for(int64_t n, int threads, int max_blocks = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

constexpr int kEnThreads = 256;
constexpr int kEnBlocks = 148 * 4;

template <int W, bool FILL>
__global__ void __launch_bounds__(256) k_pt2_gen(const uint64_t* __restrict__ keys, int64_t n,
                                                 KeyLayout L, HashView pert, ConnDev cd,
                                                 int64_t a_lo, int64_t a_hi,
                                                 int32_t* __restrict__ acount,
                                                 const int64_t* __restrict__ arowptr,
                                                 int32_t* __restrict__ ecol,
                                                 double* __restrict__ eval) {
  __shared__ uint32_t s_binom[kBinomElems];
  __shared__ uint8_t s_exc[8][128];
  fill_binom(s_binom);
  __syncthreads();
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
       i += warps) {
    uint64_t k[W];
    load_key<W>(keys, i, k);
    for_each_group<W>(cd, k, L, s_exc[threadIdx.x >> 5], s_binom, [&](int64_t u) {
      if (u < 0) return;
      const GroupDev g = cd.groups[u];
      uint64_t t[W];
      if (!group_target<W>(cd, u, g, k, L, t)) return;
      const int64_t a = hash_find<W>(pert, t, key_hash<W>(t));
      if (a < a_lo || a >= a_hi) return;
      if (!FILL) {
        atomicAdd(acount + (a - a_lo), 1);
      } else {
        const int64_t p = arowptr[a - a_lo] + atomicAdd(acount + (a - a_lo), 1);
        ecol[p] = (int32_t)i;
        eval[p] = group_value<W>(cd, g.tb, g.te, k, L);
      }
    });
  }
}

template <int W>
void pt2_count_launch(const uint64_t* keys, int64_t n, KeyLayout L, HashView pert, ConnDev cd,
                      int64_t a_lo, int64_t a_hi, int32_t* acount, cudaStream_t s) {
  note_launch(); k_pt2_gen<W, false><<<grid_for(n * 32, 256, 148 * 8), 256, 0, s>>>(
      keys, n, L, pert, cd, a_lo, a_hi, acount, nullptr, nullptr, nullptr);
}
template <int W>
void pt2_fill_launch(const uint64_t* keys, int64_t n, KeyLayout L, HashView pert, ConnDev cd,
                     int64_t a_lo, int64_t a_hi, const int64_t* arowptr, int32_t* afill,
                     int32_t* ecol, double* eval, cudaStream_t s) {
  note_launch(); k_pt2_gen<W, true><<<grid_for(n * 32, 256, 148 * 8), 256, 0, s>>>(
      keys, n, L, pert, cd, a_lo, a_hi, afill, arowptr, ecol, eval);
}

// One warp per perturber row.  Lanes own eigenvector columns n = lane + 32 r.  Each warp keeps
// running sums of num^2/(E_n - E_a) over the rows it visits; the block reduces its warps in
// fixed order into part[block][n].
template <int W, int NR>
__global__ void __launch_bounds__(kEnThreads) k_pt2_en(
    const uint64_t* __restrict__ pkeys, int64_t a_lo, int64_t a_hi, KeyLayout L, ConnDev cd,
    const int64_t* __restrict__ arowptr, const int32_t* __restrict__ ecol,
    const double* __restrict__ eval, const double* __restrict__ X, int ldx, int nopt,
    const double* __restrict__ E, double* __restrict__ part) {
  __shared__ double red[kEnThreads / 32][NR * 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  double en[NR], sum[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const int c = lane + 32 * r;
    en[r] = c < nopt ? E[c] : 0.0;
    sum[r] = 0.0;
  }
  for (int64_t a = a_lo + blockIdx.x * (int64_t)(blockDim.x >> 5) + wid; a < a_hi; a += warps) {
    double num[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) num[r] = 0.0;
    const int64_t beg = arowptr[a - a_lo], end = arowptr[a - a_lo + 1];
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
      const int64_t e = e0 + lane;
      int ii = 0;
      double hh = 0.0;
      if (e < end) { ii = ecol[e]; hh = eval[e]; }
      const int m = (int)(end - e0 < 32 ? end - e0 : 32);
#pragma unroll 4
      for (int t = 0; t < m; ++t) {
        const int i = __shfl_sync(0xffffffffu, ii, t);
        const double h = __shfl_sync(0xffffffffu, hh, t);
        const double* xr = X + (int64_t)i * ldx;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const int c = lane + 32 * r;
          if (c < nopt) num[r] = fma(h, __ldg(xr + c), num[r]);
        }
      }
    }
    double ea = 0.0;
    if (lane == 0) {
      uint64_t k[W];
      load_key<W>(pkeys, a, k);
      ea = diag_value<W>(cd, k, L);
    }
    ea = __shfl_sync(0xffffffffu, ea, 0);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int c = lane + 32 * r;
      if (c < nopt) sum[r] += (num[r] * num[r]) / (en[r] - ea);
    }
  }
#pragma unroll
  for (int r = 0; r < NR; ++r) red[wid][lane + 32 * r] = sum[r];
  __syncthreads();
  for (int c = threadIdx.x; c < nopt; c += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kEnThreads / 32; ++w) s += red[w][c];
    part[(int64_t)blockIdx.x * nopt + c] = s;
  }
}

template <int W>
void pt2_en_launch(const uint64_t* pkeys, int64_t a_lo, int64_t a_hi, KeyLayout L, ConnDev cd,
                   const int64_t* arowptr, const int32_t* ecol, const double* eval,
                   const double* X, int ldx, int nopt, const double* E, double* part,
                   cudaStream_t s) {
  switch ((nopt + 31) / 32) {
#define VHCI_EN_CASE(R)                                                                        \
  case R:                                                                                      \
    note_launch(); k_pt2_en<W, R><<<kEnBlocks, kEnThreads, 0, s>>>(pkeys, a_lo, a_hi, L, cd, arowptr, ecol, \
                                                    eval, X, ldx, nopt, E, part);            \
    break;
    VHCI_EN_CASE(1) VHCI_EN_CASE(2) VHCI_EN_CASE(3) VHCI_EN_CASE(4)
    VHCI_EN_CASE(5) VHCI_EN_CASE(6) VHCI_EN_CASE(7) VHCI_EN_CASE(8)
#undef VHCI_EN_CASE
    default: break;
  }
}

}  // namespace

void pt2_count(const uint64_t* keys, int64_t n, KeyLayout L, HashView pert, ConnDev cd,
               int64_t a_lo, int64_t a_hi, int32_t* acount, cudaStream_t s) {
  if (n <= 0) return;
  VHCI_DISPATCH_W(L.W, pt2_count_launch, keys, n, L, pert, cd, a_lo, a_hi, acount, s);
}

void pt2_fill(const uint64_t* keys, int64_t n, KeyLayout L, HashView pert, ConnDev cd,
              int64_t a_lo, int64_t a_hi, const int64_t* arowptr, int32_t* afill, int32_t* ecol,
              double* eval, cudaStream_t s) {
  if (n <= 0) return;
  VHCI_DISPATCH_W(L.W, pt2_fill_launch, keys, n, L, pert, cd, a_lo, a_hi, arowptr, afill, ecol,
                  eval, s);
}

int pt2_en_blocks() { return kEnBlocks; }

void pt2_en(const uint64_t* pkeys, int64_t a_lo, int64_t a_hi, KeyLayout L, ConnDev cd,
            const int64_t* arowptr, const int32_t* ecol, const double* eval, const double* X,
            int ldx, int nopt, const double* E, double* part, cudaStream_t s) {
  VHCI_DISPATCH_W(L.W, pt2_en_launch, pkeys, a_lo, a_hi, L, cd, arowptr, ecol, eval, X, ldx, nopt,
                  E, part, s);
}

}  // namespace vhci
