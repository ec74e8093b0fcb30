// FP64 tensor-core projections for the block Lanczos eigensolver (the Gram-Schmidt passes, the
// block orthonormalisation and the Rayleigh-Ritz rotations).  The reference eigensolver (Spectra's
// implicitly restarted Lanczos, Ham.cpp:347-370) does these with Eigen's dense products; here they
// are skinny products over the whole basis, written for B200's FP64 tensor pipe (DMMA,
// mma.sync.m8n8k4.f64), with operand tiles staged in shared memory by cp.async:
//
//   proj_gram:  C = alpha * A^T B + beta * C   A: n x M, B: n x P (row-major), C: M x P col-major
//               (P <= 16; M in slabs of 1024).  The n rows are split over the blocks; each block
//               keeps its partial slab x P product in registers (one warp per group of 8-row
//               tiles of C) and writes it to scratch; a second kernel sums the partials in block
//               order, so the result does not depend on scheduling.
//   proj_rows:  Out = alpha * A S + beta * Out   A: n x M row-major, S: M x P col-major,
//               Out: n x P row-major.  A block owns 64 rows of A (one 8-row tile per warp) and
//               streams the M dimension through shared memory in chunks of 32.
#include <algorithm>
#include <cstdint>

#include "ops.h"

namespace vhci {

namespace {

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

constexpr int kThreads = 256;
constexpr int kGramRows = 16;   // rows per shared-memory stage (four k-steps of 4)
constexpr int kGramMT = 16;     // 8-row tiles of C per warp: a slab of 8 warps x 16 x 8 = 1024
constexpr int kGramSlab = 8 * kGramMT * 8;
constexpr int kGramBlocks = 148 * 2;

// Shared row strides (doubles): roundup(M, 16) + 4 and 8 NT + 4 put the four rows of one fragment
// load into distinct 32-byte bank groups.
__host__ __device__ inline int gram_sq(int M) { return (M + 15) / 16 * 16 + 4; }

// Partial A^T B over this block's rows -> part[blockIdx.x][a][c] (M x P, a-major).  Rows are
// copied in 16-byte chunks when the pointer and stride allow it, else element by element.
// Fragment layouts of m8n8k4 (row.col): A[m][k] sits in lane 4 m + k, B[k][n] in lane 4 n + k,
// D[m][n] in lane 4 m + n / 2 (element n % 2).
template <int NT>
__global__ void __launch_bounds__(kThreads, 1) k_gram(const double* __restrict__ A, int lda,
                                                      const double* __restrict__ B, int ldb,
                                                      int64_t n, int M, int P,
                                                      double* __restrict__ part) {
  extern __shared__ double sm[];
  const int SQ = gram_sq(M);
  constexpr int SW = 8 * NT + 4;
  double* sq = sm;
  double* sw = sm + 2 * kGramRows * SQ;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = (int64_t)blockIdx.x * per, r1 = min(n, r0 + per);
  const int mt_total = (M + 7) / 8;
  double acc[kGramMT][NT][2];
#pragma unroll
  for (int t = 0; t < kGramMT; ++t)
#pragma unroll
    for (int u = 0; u < NT; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
  const int qchunks = (M + 1) / 2, bchunks = (P + 1) / 2;
  const bool va = ((lda & 1) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
  const bool vb = ((ldb & 1) == 0) && ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
  auto load = [&](int stage, int64_t i0) {
    double* dq = sq + stage * kGramRows * SQ;
    double* dw = sw + stage * kGramRows * SW;
    for (int x = threadIdx.x; x < kGramRows * qchunks; x += kThreads) {
      const int r = x / qchunks, c2 = x - r * qchunks;
      const int64_t i = i0 + r;
      double* d = dq + r * SQ + 2 * c2;
      if (va && i < r1 && 2 * c2 + 1 < M) {
        cp16(d, A + i * lda + 2 * c2);
      } else {
        d[0] = (i < r1 && 2 * c2 < M) ? A[i * lda + 2 * c2] : 0.0;
        d[1] = (i < r1 && 2 * c2 + 1 < M) ? A[i * lda + 2 * c2 + 1] : 0.0;
      }
    }
    for (int x = threadIdx.x; x < kGramRows * bchunks; x += kThreads) {
      const int r = x / bchunks, c2 = x - r * bchunks;
      const int64_t i = i0 + r;
      double* d = dw + r * SW + 2 * c2;
      if (vb && i < r1 && 2 * c2 + 1 < P) {
        cp16(d, B + i * ldb + 2 * c2);
      } else {
        d[0] = (i < r1 && 2 * c2 < P) ? B[i * ldb + 2 * c2] : 0.0;
        d[1] = (i < r1 && 2 * c2 + 1 < P) ? B[i * ldb + 2 * c2 + 1] : 0.0;
      }
    }
    cp_commit();
  };
  const int64_t nst = r1 > r0 ? (r1 - r0 + kGramRows - 1) / kGramRows : 0;
  if (nst > 0) load(0, r0);
  for (int64_t s = 0; s < nst; ++s) {
    if (s + 1 < nst) load((int)((s + 1) & 1), r0 + (s + 1) * kGramRows);
    else cp_commit();
    cp_wait1();
    __syncthreads();
    const double* dq = sq + (s & 1) * kGramRows * SQ;
    const double* dw = sw + (s & 1) * kGramRows * SW;
#pragma unroll
    for (int k = 0; k < kGramRows; k += 4) {
      const int kr = k + (lane & 3);
      double b[NT];
#pragma unroll
      for (int u = 0; u < NT; ++u) {
        const int c = 8 * u + (lane >> 2);
        b[u] = c < P ? dw[kr * SW + c] : 0.0;
      }
#pragma unroll
      for (int t = 0; t < kGramMT; ++t) {
        const int mt = wid + 8 * t;
        if (mt < mt_total) {
          const int a = 8 * mt + (lane >> 2);
          const double av = a < M ? dq[kr * SQ + a] : 0.0;
#pragma unroll
          for (int u = 0; u < NT; ++u) dmma(acc[t][u], av, b[u]);
        }
      }
    }
    __syncthreads();
  }
  double* out = part + (int64_t)blockIdx.x * M * P;
#pragma unroll
  for (int t = 0; t < kGramMT; ++t) {
    const int mt = wid + 8 * t;
    if (mt >= mt_total) continue;
    const int a = 8 * mt + (lane >> 2);
    if (a >= M) continue;
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = 8 * u + 2 * (lane & 3) + j;
        if (c < P) out[(int64_t)a * P + c] = acc[t][u][j];
      }
  }
}

__global__ void k_gram_reduce(const double* __restrict__ part, int nblk, int M, int P,
                              double alpha, double beta, double* __restrict__ C, int ldc) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < M * P; x += gridDim.x * blockDim.x) {
    const int a = x / P, c = x - a * P;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * M * P + x];
    double* o = C + a + (int64_t)c * ldc;
    *o = beta == 0.0 ? alpha * s : alpha * s + beta * *o;
  }
}

constexpr int kRowsTile = 64, kRowsKC = 32;

template <int NT>
constexpr size_t rows_smem() {
  return (size_t)(2 * kRowsTile * (kRowsKC + 4) + 2 * kRowsKC * (8 * NT + 4)) * sizeof(double);
}

// Out[i][c] = alpha sum_a A[i][a] S[a + c lds] + beta Out[i][c] for 64 rows and up to 8 NT
// columns.  Shared memory: two stages of the A tile (64 x 36) and of the S tile (32 x 8 NT + 4).
template <int NT>
__global__ void __launch_bounds__(kThreads) k_rows(const double* __restrict__ A, int lda,
                                                   const double* __restrict__ S, int lds,
                                                   int64_t n, int M, int P, double alpha,
                                                   double beta, double* __restrict__ Out,
                                                   int ldo) {
  extern __shared__ double smr[];
  auto sa = reinterpret_cast<double(*)[kRowsTile][kRowsKC + 4]>(smr);
  auto ss = reinterpret_cast<double(*)[kRowsKC][8 * NT + 4]>(smr + 2 * kRowsTile * (kRowsKC + 4));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t i0 = (int64_t)blockIdx.x * kRowsTile;
  double acc[NT][2];
#pragma unroll
  for (int u = 0; u < NT; ++u) acc[u][0] = acc[u][1] = 0.0;
  const int nk = (M + kRowsKC - 1) / kRowsKC;
  const bool vec = ((lda & 1) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
  auto load = [&](int stage, int k0) {
    for (int x = threadIdx.x; x < kRowsTile * (kRowsKC / 2); x += kThreads) {
      const int r = x / (kRowsKC / 2), c2 = x - r * (kRowsKC / 2);
      const int64_t i = i0 + r;
      const int a = k0 + 2 * c2;
      double* d = &sa[stage][r][2 * c2];
      if (vec && i < n && a + 1 < M) {
        cp16(d, A + i * lda + a);
      } else {
        d[0] = (i < n && a < M) ? A[i * lda + a] : 0.0;
        d[1] = (i < n && a + 1 < M) ? A[i * lda + a + 1] : 0.0;
      }
    }
    for (int x = threadIdx.x; x < kRowsKC * 8 * NT; x += kThreads) {
      const int r = x / (8 * NT), c = x - r * (8 * NT);
      const int a = k0 + r;
      ss[stage][r][c] = (a < M && c < P) ? S[a + (int64_t)c * lds] : 0.0;
    }
    cp_commit();
  };
  load(0, 0);
  for (int kc = 0; kc < nk; ++kc) {
    if (kc + 1 < nk) load((kc + 1) & 1, (kc + 1) * kRowsKC);
    else cp_commit();
    cp_wait1();
    __syncthreads();
    const int st = kc & 1;
#pragma unroll
    for (int k = 0; k < kRowsKC; k += 4) {
      const double av = sa[st][8 * wid + (lane >> 2)][k + (lane & 3)];
#pragma unroll
      for (int u = 0; u < NT; ++u) dmma(acc[u], av, ss[st][k + (lane & 3)][8 * u + (lane >> 2)]);
    }
    __syncthreads();
  }
  const int64_t i = i0 + 8 * wid + (lane >> 2);
  if (i < n) {
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = 8 * u + 2 * (lane & 3) + j;
        if (c < P) {
          double* o = Out + i * ldo + c;
          *o = beta == 0.0 ? alpha * acc[u][j] : alpha * acc[u][j] + beta * *o;
        }
      }
  }
}

}  // namespace

int64_t proj_gram_scratch(int M, int P) {
  return (int64_t)kGramBlocks * std::min(M, kGramSlab) * P;
}

bool proj_gram(const double* A, int lda, const double* B, int ldb, int64_t n, int M, int P,
               double alpha, double beta, double* C, int ldc, double* part, cudaStream_t s) {
  if (M <= 0 || P <= 0) return true;
  if (P > 16 || lda < M || ldb < P) return false;
  const int NT = P <= 8 ? 1 : 2;
  int nblk = kGramBlocks;
  if (n < (int64_t)nblk * kGramRows)
    nblk = (int)std::max<int64_t>(1, (n + kGramRows - 1) / kGramRows);
  for (int a0 = 0; a0 < M; a0 += kGramSlab) {
    const int Mc = std::min(kGramSlab, M - a0);
    const int SQ = gram_sq(Mc);
    const size_t smem =
        (size_t)(2 * kGramRows * SQ + 2 * kGramRows * (8 * NT + 4)) * sizeof(double);
    note_launch();
    if (NT == 1) {
      cudaFuncSetAttribute(k_gram<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_gram<1><<<nblk, kThreads, smem, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
    } else {
      cudaFuncSetAttribute(k_gram<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_gram<2><<<nblk, kThreads, smem, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
    }
    note_launch();
    k_gram_reduce<<<(Mc * P + 255) / 256, 256, 0, s>>>(part, nblk, Mc, P, alpha, beta, C + a0,
                                                        ldc);
  }
  return true;
}

void proj_rows(const double* A, int lda, const double* S, int lds, int64_t n, int M, int P,
               double alpha, double beta, double* Out, int ldo, cudaStream_t s) {
  if (n <= 0 || P <= 0) return;
  const unsigned g = (unsigned)((n + kRowsTile - 1) / kRowsTile);
  for (int c0 = 0; c0 < P; c0 += 64) {
    const int pc = std::min(64, P - c0);
    const double* Sc = S + (int64_t)c0 * lds;
    double* Oc = Out + c0;
    note_launch();
#define VHCI_ROWS(NTV)                                                                          \
  do {                                                                                          \
    cudaFuncSetAttribute(k_rows<NTV>, cudaFuncAttributeMaxDynamicSharedMemorySize,              \
                         (int)rows_smem<NTV>());                                                \
    k_rows<NTV><<<g, kThreads, rows_smem<NTV>(), s>>>(A, lda, Sc, lds, n, M, pc, alpha, beta,  \
                                                      Oc, ldo);                                 \
  } while (0)
    if (pc <= 8) VHCI_ROWS(1);
    else if (pc <= 16) VHCI_ROWS(2);
    else if (pc <= 32) VHCI_ROWS(4);
    else VHCI_ROWS(8);
#undef VHCI_ROWS
  }
}

}  // namespace vhci
