// Epstein-Nesbet PT2 kernels (reference: DoPT2, PT2.cpp:16-154).
//
// The reference loops over every (perturber a, variational state i) pair.  Here the connected
// pairs are generated from the variational side: for each state i and connection group u, the
// target a = i + Delta_u is looked up in the perturber hash; hits become entries (a, i, H_ai) of a
// perturber-row CSR (count pass, scan, fill pass).  A fused kernel then forms
// num_a[n] = sum_i H_ai C_in, E_a = H_aa, and sum_a num_a[n]^2 / (E_n - E_a) per block.
#include <climits>

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
    const double* __restrict__ E, double* __restrict__ part, int ldp) {
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
    part[(int64_t)blockIdx.x * ldp + c] = s;
  }
}

// The EN kernel holds NR <= 8 columns per lane, i.e. at most 256 eigenvector columns; wider
// requests (Nstate > 256; the reference has no such limit, PT2.cpp:29-37) run as column tiles of
// 256, each tile writing its own columns of `part` (leading dimension nopt).
constexpr int kEnMaxCols = 8 * 32;

template <int W>
bool pt2_en_launch(const uint64_t* pkeys, int64_t a_lo, int64_t a_hi, KeyLayout L, ConnDev cd,
                   const int64_t* arowptr, const int32_t* ecol, const double* eval,
                   const double* X, int ldx, int nopt, const double* E, double* part,
                   cudaStream_t s) {
  for (int c0 = 0; c0 < nopt; c0 += kEnMaxCols) {
    const int nc = nopt - c0 < kEnMaxCols ? nopt - c0 : kEnMaxCols;
    switch ((nc + 31) / 32) {
#define VHCI_EN_CASE(R)                                                                        \
  case R:                                                                                      \
    note_launch();                                                                             \
    k_pt2_en<W, R><<<kEnBlocks, kEnThreads, 0, s>>>(pkeys, a_lo, a_hi, L, cd, arowptr, ecol,  \
                                                    eval, X + c0, ldx, nc, E + c0, part + c0, \
                                                    nopt);                                     \
    break;
      VHCI_EN_CASE(1) VHCI_EN_CASE(2) VHCI_EN_CASE(3) VHCI_EN_CASE(4)
      VHCI_EN_CASE(5) VHCI_EN_CASE(6) VHCI_EN_CASE(7) VHCI_EN_CASE(8)
#undef VHCI_EN_CASE
      default:
        return false;
    }
  }
  return true;
}

// ---- fixed entry order within perturber rows --------------------------------------------------
// The fill pass takes slots with atomics, so the order of a row's entries (and with it the FP64
// summation order of num_a) would change from run to run.  Each (a, i) pair occurs once per row
// (distinct connection groups move i to distinct targets), so sorting a row by i gives one
// canonical order, and the EN sums become reproducible bit for bit.

constexpr int kSortWarpCap = 256;  // rows up to this length: one warp, shared-memory bitonic sort

// Bitonic sort of the row held one entry per lane (m <= 32; padding keys are INT_MAX).
__device__ __forceinline__ void warp_bitonic(int& key, double& v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int ok = __shfl_xor_sync(0xffffffffu, key, j);
      const double ov = __shfl_xor_sync(0xffffffffu, v, j);
      const bool up = (lane & k) == 0, lower = (lane & j) == 0;
      const bool take = lower ? (up ? ok < key : ok > key) : (up ? ok > key : ok < key);
      if (take) { key = ok; v = ov; }
    }
  }
}

// One warp per row for rows of 2..kSortWarpCap entries; longer rows are left to k_pt2_sort_long.
__global__ void __launch_bounds__(256) k_pt2_sort_rows(const int64_t* __restrict__ arowptr,
                                                       int64_t nrows, int32_t* __restrict__ ecol,
                                                       double* __restrict__ eval) {
  __shared__ int32_t sk[8][kSortWarpCap];
  __shared__ double sv[8][kSortWarpCap];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + wid; r < nrows; r += warps) {
    const int64_t beg = arowptr[r], end = arowptr[r + 1];
    const int m = (int)(end - beg);
    if (m <= 1 || m > kSortWarpCap) continue;
    if (m <= 32) {
      int key = lane < m ? ecol[beg + lane] : INT_MAX;
      double v = lane < m ? eval[beg + lane] : 0.0;
      warp_bitonic(key, v);
      if (lane < m) { ecol[beg + lane] = key; eval[beg + lane] = v; }
      continue;
    }
    int P = 64;
    while (P < m) P <<= 1;
    for (int t = lane; t < P; t += 32) {
      sk[wid][t] = t < m ? ecol[beg + t] : INT_MAX;
      sv[wid][t] = t < m ? eval[beg + t] : 0.0;
    }
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = lane; t < P; t += 32) {
          const int u = t ^ j;
          if (u > t) {
            const int a = sk[wid][t], b = sk[wid][u];
            if ((a > b) == ((t & k) == 0)) {
              sk[wid][t] = b; sk[wid][u] = a;
              const double x = sv[wid][t]; sv[wid][t] = sv[wid][u]; sv[wid][u] = x;
            }
          }
        }
        __syncwarp();
      }
    for (int t = lane; t < m; t += 32) { ecol[beg + t] = sk[wid][t]; eval[beg + t] = sv[wid][t]; }
    __syncwarp();
  }
}

// One block per long row (rows[] lists them): the row is copied to scratch (tcol, tval at the
// row's offset in the scratch, soff), then every entry goes to position beg + rank, its rank
// being the number of smaller i in the row (the i are distinct).  Cost m^2 / blockDim per row.
__global__ void __launch_bounds__(256) k_pt2_sort_long(const int64_t* __restrict__ arowptr,
                                                       const int64_t* __restrict__ rows,
                                                       const int64_t* __restrict__ soff,
                                                       int32_t* __restrict__ ecol,
                                                       double* __restrict__ eval,
                                                       int32_t* __restrict__ tcol,
                                                       double* __restrict__ tval) {
  __shared__ int32_t tile[2048];
  const int64_t r = rows[blockIdx.x];
  const int64_t beg = arowptr[r], m = arowptr[r + 1] - beg;
  int32_t* tc = tcol + soff[blockIdx.x];
  double* tv = tval + soff[blockIdx.x];
  for (int64_t t = threadIdx.x; t < m; t += blockDim.x) { tc[t] = ecol[beg + t]; tv[t] = eval[beg + t]; }
  __syncthreads();
  for (int64_t t0 = 0; t0 < m; t0 += blockDim.x) {
    const int64_t t = t0 + threadIdx.x;
    const int mine = t < m ? tc[t] : INT_MAX;
    int64_t rank = 0;
    for (int64_t q0 = 0; q0 < m; q0 += 2048) {
      const int qn = (int)(m - q0 < 2048 ? m - q0 : 2048);
      __syncthreads();
      for (int q = threadIdx.x; q < qn; q += blockDim.x) tile[q] = tc[q0 + q];
      __syncthreads();
      for (int q = 0; q < qn; ++q) rank += tile[q] < mine;
    }
    if (t < m) { ecol[beg + rank] = mine; eval[beg + rank] = tv[t]; }
  }
}

// crow[i] = arow[i] - arow[0], i in [0, nrows]: a chunk's row offsets from the whole range's.
__global__ void k_pt2_rebase(const int64_t* __restrict__ arow, int64_t nrows,
                             int64_t* __restrict__ crow) {
  const int64_t base = arow[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= nrows;
       i += (int64_t)gridDim.x * blockDim.x)
    crow[i] = arow[i] - base;
}

// Lists the rows of at least minlen entries: rows[q] and a disjoint scratch offset soff[q] of
// the row's length, q from an atomic counter (cnt[0] rows, cnt[1] entries).  The order of the
// list does not matter: each listed row is ordered by its own block.
__global__ void k_pt2_list_long(const int64_t* __restrict__ arowptr, int64_t nrows, int minlen,
                                int64_t* __restrict__ rows, int64_t* __restrict__ soff,
                                unsigned long long* __restrict__ cnt) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t len = arowptr[r + 1] - arowptr[r];
    if (len >= minlen) {
      const unsigned long long q = atomicAdd(cnt, 1ull);
      rows[q] = r;
      soff[q] = (int64_t)atomicAdd(cnt + 1, (unsigned long long)len);
    }
  }
}

}  // namespace

void pt2_rebase_rows(const int64_t* arow, int64_t nrows, int64_t* crow, cudaStream_t s) {
  note_launch();
  k_pt2_rebase<<<grid_for(nrows + 1, 256, 148 * 8), 256, 0, s>>>(arow, nrows, crow);
}

void pt2_list_long(const int64_t* arowptr, int64_t nrows, int64_t* rows, int64_t* soff,
                   unsigned long long* cnt, cudaStream_t s) {
  if (nrows <= 0) return;
  note_launch();
  k_pt2_list_long<<<grid_for(nrows, 256, 148 * 8), 256, 0, s>>>(arowptr, nrows, kSortWarpCap + 1,
                                                                 rows, soff, cnt);
}

void pt2_sort_rows(const int64_t* arowptr, int64_t nrows, int32_t* ecol, double* eval,
                   cudaStream_t s) {
  if (nrows <= 0) return;
  note_launch();
  k_pt2_sort_rows<<<grid_for(nrows * 32, 256, 148 * 8), 256, 0, s>>>(arowptr, nrows, ecol, eval);
}

int pt2_sort_long_min() { return kSortWarpCap + 1; }

void pt2_sort_long(const int64_t* arowptr, const int64_t* rows, const int64_t* soff, int nlong,
                   int32_t* ecol, double* eval, int32_t* tcol, double* tval, cudaStream_t s) {
  if (nlong <= 0) return;
  note_launch();
  k_pt2_sort_long<<<nlong, 256, 0, s>>>(arowptr, rows, soff, ecol, eval, tcol, tval);
}

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

bool pt2_en(const uint64_t* pkeys, int64_t a_lo, int64_t a_hi, KeyLayout L, ConnDev cd,
            const int64_t* arowptr, const int32_t* ecol, const double* eval, const double* X,
            int ldx, int nopt, const double* E, double* part, cudaStream_t s) {
  if (nopt <= 0) return false;
  switch (L.W) {
#define VHCI_EN_W(WV) \
  case WV: return pt2_en_launch<WV>(pkeys, a_lo, a_hi, L, cd, arowptr, ecol, eval, X, ldx, nopt, E, part, s);
    VHCI_EN_W(1) VHCI_EN_W(2) VHCI_EN_W(3) VHCI_EN_W(4)
    VHCI_EN_W(5) VHCI_EN_W(6) VHCI_EN_W(7) VHCI_EN_W(8)
#undef VHCI_EN_W
    default: return false;
  }
}

}  // namespace vhci
