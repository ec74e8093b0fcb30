// FP64 tensor-core projections for the block Lanczos eigensolver (the Gram-Schmidt passes, the
// block orthonormalisation and the Rayleigh-Ritz rotations).  The reference eigensolver (Spectra's
// implicitly restarted Lanczos, Ham.cpp:347-370) does these with Eigen's dense products; here they
// are skinny products over the whole basis, written for B200's FP64 tensor pipe (DMMA,
// mma.sync.m8n8k4.f64).  Both read the tall operand once, straight from global memory into the
// DMMA fragment registers (each lane's fragment element is 8 bytes of a 32-byte row segment, so
// the sectors are fully used), with several k-steps of loads in flight per lane and 32 warps per
// SM; the main loops have no block-wide barriers:
//
//   proj_gram:  C = alpha * A^T B + beta * C   A: n x M, B: n x P (row-major), C: M x P col-major,
//               P <= 16.  A persistent grid splits the n rows over the blocks; each warp keeps
//               the partial products of its 8-row tiles of C in registers; the blocks' partials
//               go to scratch and a second kernel sums them in block order, so the result does not
//               depend on scheduling.
//   proj_rows:  Out = alpha * A S + beta * Out   A: n x M row-major, S: M x P col-major,
//               Out: n x P row-major.  Each block holds a 16-column slab of S in shared memory
//               and its warps stream 8-row tiles of A.
//
// Fragment layouts of m8n8k4 (row.col): A[m][k] sits in lane 4 m + k, B[k][n] in lane 4 n + k,
// D[m][n] in lane 4 m + n / 2 (element n % 2).
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "ops.h"

namespace vhci {

namespace {

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

constexpr int kThreads = 1024;      // proj_rows: 32 warps, one block per SM
constexpr int kBlocks = 148;
constexpr int kUnroll = 8;          // proj_rows: k-steps of loads issued ahead
constexpr int kGramThreads = 512;   // proj_gram: 16 warps with up to 128 registers each
constexpr int kGramWarps = kGramThreads / 32;
constexpr int kGramTiles = 6;       // 8-row tiles of C per warp: a slab of 16 x 6 x 8 = 768 rows
constexpr int kGramSlab = kGramWarps * kGramTiles * 8;
constexpr int kGramUnroll = 2;

// Partial A^T B over this block's rows for the columns a0 .. a0 + Mc - 1 of A.  The 8-row tiles
// of C are dealt to a group of WG = ceil(tiles / TILES) warps (warp g of a group owns tiles g,
// g + WG, ...); the block's 16 warps form 16 / WG such groups, which take turns over the block's
// rows in steps of 4 UNROLL rows, so a narrow C (few tiles) still keeps every warp streaming.
// When a group would need more than half the warps, all 16 form one group.
// Group r of block x writes its partial to part[x * groups + r] (Mc x P, a-major).
template <int NT, int TILES, int UNROLL, int NWARP>
__global__ void __launch_bounds__(NWARP * 32, 1) k_gram(const double* __restrict__ A, int lda,
                                                    const double* __restrict__ B, int ldb,
                                                    int64_t n, int Mc, int P,
                                                    double* __restrict__ part) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int mt_total = (Mc + 7) / 8;
  int WG = (mt_total + TILES - 1) / TILES;
  if (2 * WG > NWARP) WG = NWARP;  // one group: spread the tiles over all warps
  const int RG = NWARP / WG;
  const int rg = wid / WG, wg = wid - rg * WG;
  if (rg >= RG) return;
  const int64_t per = ((n + gridDim.x - 1) / gridDim.x + 3) & ~int64_t(3);
  const int64_t r0 = (int64_t)blockIdx.x * per, r1 = min(n, r0 + per);
  double acc[TILES][NT][2];
#pragma unroll
  for (int t = 0; t < TILES; ++t)
#pragma unroll
    for (int u = 0; u < NT; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
  int acol[TILES];
  bool aon[TILES];
#pragma unroll
  for (int t = 0; t < TILES; ++t) {
    acol[t] = 8 * (wg + WG * t) + (lane >> 2);
    aon[t] = (wg + WG * t) < mt_total && acol[t] < Mc;
  }
  const int kl = lane & 3;
  for (int64_t k0 = r0 + 4 * UNROLL * rg; k0 < r1; k0 += 4 * UNROLL * RG) {
    double a[UNROLL][TILES], b[UNROLL][NT];
#pragma unroll
    for (int s = 0; s < UNROLL; ++s) {
      const int64_t i = k0 + 4 * s + kl;
      const bool rin = i < r1;
#pragma unroll
      for (int t = 0; t < TILES; ++t)
        a[s][t] = (rin && aon[t]) ? __ldg(A + i * lda + acol[t]) : 0.0;
#pragma unroll
      for (int u = 0; u < NT; ++u) {
        const int c = 8 * u + (lane >> 2);
        b[s][u] = (rin && c < P) ? __ldg(B + i * ldb + c) : 0.0;
      }
    }
#pragma unroll
    for (int s = 0; s < UNROLL; ++s)
#pragma unroll
      for (int t = 0; t < TILES; ++t)
        if ((wg + WG * t) < mt_total)
#pragma unroll
          for (int u = 0; u < NT; ++u) dmma(acc[t][u], a[s][t], b[s][u]);
  }
  double* out = part + ((int64_t)blockIdx.x * RG + rg) * Mc * P;
#pragma unroll
  for (int t = 0; t < TILES; ++t) {
    const int mt = wg + WG * t;
    if (mt >= mt_total) continue;
    const int r = 8 * mt + (lane >> 2);
    if (r >= Mc) continue;
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = 8 * u + 2 * (lane & 3) + j;
        if (c < P) out[(int64_t)r * P + c] = acc[t][u][j];
      }
  }
}

// Row groups of one k_gram launch (as the kernel computes them).
inline int gram_groups(int Mc, int tiles_per_warp, int nwarp) {
  const int mt = (Mc + 7) / 8;
  const int wg = (mt + tiles_per_warp - 1) / tiles_per_warp;
  return 2 * wg > nwarp ? 1 : nwarp / wg;
}

// Sums the blocks' partials: a block of kRedWarps warps owns 32 consecutive entries of C; warp w
// adds the partials of blocks w, w + kRedWarps, ... (lane = entry, so each partial row is read as
// one 256-byte segment) and the warps' sums are combined in warp order, so the result is the same
// on every run.  32 warps: a narrow product leaves thousands of partials (148 blocks x 16 row
// groups) for few entries of C.
constexpr int kRedWarps = 32;
__global__ void __launch_bounds__(kRedWarps * 32) k_gram_reduce(const double* __restrict__ part,
                                                                int nblk, int M, int P, double alpha,
                                                                double beta, double* __restrict__ C,
                                                                int ldc) {
  __shared__ double ws[kRedWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = blockIdx.x * 32 + lane;
  const int64_t mp = (int64_t)M * P;
  double s = 0.0;
  if (x < mp)
    for (int b = w; b < nblk; b += kRedWarps) s += part[b * mp + x];
  ws[w][lane] = s;
  __syncthreads();
  if (w == 0 && x < mp) {
    double t = ws[0][lane];
#pragma unroll
    for (int v = 1; v < kRedWarps; ++v) t += ws[v][lane];
    const int a = x / P, c = x - a * P;
    double* o = C + a + (int64_t)c * ldc;
    *o = beta == 0.0 ? alpha * t : alpha * t + beta * *o;
  }
}

// Shared row stride of the S slab: 8 NT + 4 doubles puts the four k-rows of one fragment load into
// distinct 32-byte bank groups.
constexpr int kRowsMaxM = 1280;     // rows of S held in shared memory per pass over A
constexpr int kRowsMaxM4 = 768;     // the same for 32-column slabs

template <int NT>
constexpr size_t rows_smem(int M) {
  return (size_t)M * (8 * NT + 4) * sizeof(double);
}

// Out[i][c] = alpha sum_a A[i][a] S[a + c lds] + beta Out[i][c] for the Mc rows of S starting
// at a0 (accum: add this slab to Out, which already holds the earlier slabs' sum; the alpha/beta
// update happens on the first slab).  Warps stream 8-row tiles of A over the whole grid.
template <int NT>
__global__ void __launch_bounds__(kThreads, 1) k_rows(const double* __restrict__ A, int lda,
                                                      const double* __restrict__ S, int lds,
                                                      int64_t n, int Mc, int P, double alpha,
                                                      double beta, double* __restrict__ Out,
                                                      int ldo) {
  extern __shared__ double ss[];  // [Mc][8 NT + 4]
  constexpr int SW = 8 * NT + 4;
  for (int x = threadIdx.x; x < Mc * 8 * NT; x += blockDim.x) {
    const int a = x / (8 * NT), c = x - a * (8 * NT);
    ss[a * SW + c] = c < P ? S[a + (int64_t)c * lds] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int kl = lane & 3;
  const int64_t tiles = (n + 7) / 8;
  const int64_t wstride = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile < tiles;
       tile += wstride) {
    const int64_t i = tile * 8 + (lane >> 2);
    const bool rin = i < n;
    const double* arow = A + (rin ? i : 0) * lda;
    double acc[NT][2];
#pragma unroll
    for (int u = 0; u < NT; ++u) acc[u][0] = acc[u][1] = 0.0;
    for (int k0 = 0; k0 < Mc; k0 += 4 * kUnroll) {
      double a[kUnroll];
#pragma unroll
      for (int s = 0; s < kUnroll; ++s) {
        const int k = k0 + 4 * s + kl;
        a[s] = (rin && k < Mc) ? __ldg(arow + k) : 0.0;
      }
#pragma unroll
      for (int s = 0; s < kUnroll; ++s) {
        const int k = k0 + 4 * s + kl;
        if (k0 + 4 * s < Mc) {
#pragma unroll
          for (int u = 0; u < NT; ++u)
            dmma(acc[u], a[s], k < Mc ? ss[k * SW + 8 * u + (lane >> 2)] : 0.0);
        }
      }
    }
    if (rin) {
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
}

// The second and third Gram-Schmidt passes over the same rows of A, fused:
//   W <- W - A S1            (S1: M x P column-major)
//   part[block] = A^T W      (with the updated W; this block's rows, M x P a-major)
// A block walks chunks of 128 rows (16 8-row tiles): warps w and w + 16 each form the product of
// tile w over one half of A's columns (A from global memory, S1 from shared memory), the second
// hands its half to the first through shared memory, which updates the tile of W and leaves the
// new rows in a shared copy; then every warp adds A_chunk^T W_chunk to its 8-row tiles of the
// partial Gram product, re-reading the chunk's rows of A, which the first phase has just brought
// into L2.  One pass over A from HBM instead of two: the chunks in flight over the whole GPU
// (148 x 128 rows of A, 58 MB at M = 384, 97 MB at M = 640) stay within L2, which 256-row chunks
// did not (measured: 31 % L2 hits on the re-read at M = 437 with 256-row chunks).
constexpr int kFuseChunk = 128;
constexpr int kFuseTiles = 3;       // Gram tiles per warp: M <= 32 x 3 x 8 = 768
constexpr int kFuseMaxM = 32 * kFuseTiles * 8;

template <int NT>
constexpr size_t fuse_smem(int M) {
  // S1 slab, chunk of W, and the second half-products of phase 1 (16 warps x 32 lanes x NT x 2)
  return (size_t)(M + kFuseChunk) * (8 * NT + 4) * sizeof(double) +
         (size_t)16 * 32 * NT * 2 * sizeof(double);
}

template <int NT>
__global__ void __launch_bounds__(kThreads, 1) k_rows_gram(const double* __restrict__ A, int lda,
                                                           const double* __restrict__ S1, int lds,
                                                           double* __restrict__ W, int ldw,
                                                           int64_t n, int M, int P,
                                                           double* __restrict__ part) {
  extern __shared__ double smf[];
  constexpr int SW = 8 * NT + 4;
  double* sS = smf;               // [M][SW]
  double* sW = smf + M * SW;      // [kFuseChunk][SW]
  double* sH = sW + kFuseChunk * SW;  // [16][32][NT][2]: phase-1 products of the upper warps
  for (int x = threadIdx.x; x < M * 8 * NT; x += blockDim.x) {
    const int a = x / (8 * NT), c = x - a * (8 * NT);
    sS[a * SW + c] = c < P ? S1[a + (int64_t)c * lds] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, kl = lane & 3;
  const int64_t per = ((n + gridDim.x - 1) / gridDim.x + 3) & ~int64_t(3);
  const int64_t r0 = (int64_t)blockIdx.x * per, r1 = min(n, r0 + per);
  const int mt_total = (M + 7) / 8;
  double g[kFuseTiles][NT][2];
#pragma unroll
  for (int t = 0; t < kFuseTiles; ++t)
#pragma unroll
    for (int u = 0; u < NT; ++u) g[t][u][0] = g[t][u][1] = 0.0;
  for (int64_t c0 = r0; c0 < r1; c0 += kFuseChunk) {
    // phase 1: tile wid % 16 of W - A S1; warps 0-15 take A's columns [0, kh), warps 16-31
    // [kh, M), kh a multiple of the 4 kUnroll columns one step covers
    const int tl = wid & 15, half = wid >> 4;
    const int kh = ((M + 1) / 2 + 4 * kUnroll - 1) / (4 * kUnroll) * (4 * kUnroll);
    const int kb = half ? kh : 0, ke = half ? M : min(kh, M);
    const int64_t i = c0 + 8 * tl + (lane >> 2);
    const bool rin = i < r1;
    const double* arow = A + (rin ? i : 0) * lda;
    double acc[NT][2];
#pragma unroll
    for (int u = 0; u < NT; ++u) acc[u][0] = acc[u][1] = 0.0;
    for (int k0 = kb; k0 < ke; k0 += 4 * kUnroll) {
      double a[kUnroll];
#pragma unroll
      for (int s = 0; s < kUnroll; ++s) {
        const int k = k0 + 4 * s + kl;
        a[s] = (rin && k < ke) ? __ldg(arow + k) : 0.0;
      }
#pragma unroll
      for (int s = 0; s < kUnroll; ++s) {
        const int k = k0 + 4 * s + kl;
        if (k0 + 4 * s < ke) {
#pragma unroll
          for (int u = 0; u < NT; ++u)
            dmma(acc[u], a[s], k < ke ? sS[k * SW + 8 * u + (lane >> 2)] : 0.0);
        }
      }
    }
    if (half) {
#pragma unroll
      for (int u = 0; u < NT; ++u)
#pragma unroll
        for (int j = 0; j < 2; ++j) sH[((tl * 32 + lane) * NT + u) * 2 + j] = acc[u][j];
    }
    __syncthreads();
    const int rl = 8 * tl + (lane >> 2);
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = 8 * u + 2 * (lane & 3) + j;
        if (half) continue;
        double wv = 0.0;
        if (rin && c < P) {
          wv = W[i * ldw + c] - (acc[u][j] + sH[((tl * 32 + lane) * NT + u) * 2 + j]);
          W[i * ldw + c] = wv;
        }
        sW[rl * SW + c] = wv;
      }
    __syncthreads();
    // phase 2: the partial Gram product of the chunk, this warp's tiles w, w + 32, w + 64
    for (int kk = 0; kk < kFuseChunk; kk += 8) {
      double a[2][kFuseTiles], b[2][NT];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int kr = kk + 4 * s + kl;
        const int64_t ir = c0 + kr;
        const bool in2 = ir < r1;
#pragma unroll
        for (int t = 0; t < kFuseTiles; ++t) {
          const int col = 8 * (wid + 32 * t) + (lane >> 2);
          a[s][t] = (in2 && col < M) ? __ldg(A + ir * lda + col) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < NT; ++u) b[s][u] = sW[kr * SW + 8 * u + (lane >> 2)];
      }
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int t = 0; t < kFuseTiles; ++t)
          if (wid + 32 * t < mt_total)
#pragma unroll
            for (int u = 0; u < NT; ++u) dmma(g[t][u], a[s][t], b[s][u]);
    }
    __syncthreads();
  }
  double* out = part + (int64_t)blockIdx.x * M * P;
#pragma unroll
  for (int t = 0; t < kFuseTiles; ++t) {
    const int mt = wid + 32 * t;
    if (mt >= mt_total) continue;
    const int r = 8 * mt + (lane >> 2);
    if (r >= M) continue;
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = 8 * u + 2 * (lane & 3) + j;
        if (c < P) out[(int64_t)r * P + c] = g[t][u][j];
      }
  }
}

// SVQB factor of a small Gram matrix on the device (one block of 128 threads), so that a Lanczos
// step needs no host round trip.  S (nb x nb, column-major, nb <= 16) = W^T W.  With
// D = diag(S)^(-1/2) (zero for a diagonal at or below 1e-28 of the largest), D S D = U L U^T by
// cyclic Jacobi in the parallel round-robin order (nb/2 disjoint rotations per round, Golub-Van
// Loan's symmetric 2 x 2 Schur step; one thread per (rotation, row) update), at most 30 sweeps,
// stopping when every off-diagonal |a_ij| <= 1e-14 sqrt(a_ii a_jj) among the directions above
// 1e-12 of the largest (the relative test bounds the orthonormality of W M independently of the
// block's conditioning); the directions with L > 1e-12 max(L) are kept in descending order and
// M[:, q] = D U[:, keep_q] / sqrt(L[keep_q]) (columns past the rank are zero).  W M is then
// orthonormal.  *rank_short is set to 1 when fewer than nb directions are kept.
constexpr int kSvqbThreads = 128;
__global__ void __launch_bounds__(kSvqbThreads) k_svqb_factor(const double* __restrict__ S, int nb,
                                                              double* __restrict__ M,
                                                              int* __restrict__ rank_short) {
  __shared__ double A[16][17], U[16][17], d[16], cs[8], sn[8], red[kSvqbThreads / 32];
  __shared__ int pa[8], pb[8], keep[16];
  __shared__ int stop, rr;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int x = tid; x < nb * nb; x += kSvqbThreads) A[x % nb][x / nb] = S[x];
  __syncthreads();
  if (tid == 0) {
    double dmax = 0.0;
    for (int i = 0; i < nb; ++i) dmax = fmax(dmax, A[i][i]);
    for (int i = 0; i < nb; ++i) {
      const double v = A[i][i];
      d[i] = (v > 1e-28 * dmax && v > 1e-300) ? 1.0 / sqrt(v) : 0.0;
    }
  }
  __syncthreads();
  for (int x = tid; x < 256; x += kSvqbThreads) {
    const int i = x & 15, j = x >> 4;
    if (i < nb && j < nb) {
      A[i][j] *= d[i] * d[j];
      U[i][j] = i == j ? 1.0 : 0.0;
    }
  }
  __syncthreads();
  const int N = (nb + 1) & ~1;  // players of the round-robin (one idle index when nb is odd)
  for (int sweep = 0; sweep < 30; ++sweep) {
    // relative off-diagonal size over the directions that count
    double dmx = 0.0;
    for (int i = 0; i < nb; ++i) dmx = fmax(dmx, A[i][i]);
    double mr = 0.0;
    for (int x = tid; x < 256; x += kSvqbThreads) {
      const int i = x & 15, j = x >> 4;
      if (i < j && j < nb && A[i][i] > 1e-12 * dmx && A[j][j] > 1e-12 * dmx)
        mr = fmax(mr, fabs(A[i][j]) / sqrt(A[i][i] * A[j][j]));
    }
    for (int o = 16; o > 0; o >>= 1) mr = fmax(mr, __shfl_xor_sync(~0u, mr, o));
    if (lane == 0) red[wid] = mr;
    __syncthreads();
    if (tid == 0) {
      double m = 0.0;
      for (int w = 0; w < kSvqbThreads / 32; ++w) m = fmax(m, red[w]);
      stop = m <= 1e-14 ? 1 : 0;
    }
    __syncthreads();
    if (stop) break;
    for (int round = 0; round < N - 1; ++round) {
      if (tid < N / 2) {
        int a = tid == 0 ? N - 1 : (tid + round) % (N - 1);
        int b = tid == 0 ? round % (N - 1) : (N - 1 - tid + round) % (N - 1);
        if (a > b) { const int t = a; a = b; b = t; }
        double c = 1.0, sg = 0.0;
        if (b < nb) {
          const double apq = A[a][b];
          if (fabs(apq) >= 1e-300) {
            const double theta = (A[b][b] - A[a][a]) / (2.0 * apq);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            sg = t * c;
          }
        }
        pa[tid] = a; pb[tid] = b; cs[tid] = c; sn[tid] = sg;
      }
      __syncthreads();
      const int t = tid >> 4, k = tid & 15;  // rotation t, row / column k
      const bool on = t < N / 2 && k < nb && pb[t] < nb;
      if (on) {  // rows a, b
        const int a = pa[t], b = pb[t];
        const double ra = A[a][k], rb = A[b][k];
        A[a][k] = cs[t] * ra - sn[t] * rb;
        A[b][k] = sn[t] * ra + cs[t] * rb;
      }
      __syncthreads();
      if (on) {  // columns a, b of A and U
        const int a = pa[t], b = pb[t];
        const double ca = A[k][a], cb = A[k][b];
        A[k][a] = cs[t] * ca - sn[t] * cb;
        A[k][b] = sn[t] * ca + cs[t] * cb;
        const double ua = U[k][a], ub = U[k][b];
        U[k][a] = cs[t] * ua - sn[t] * ub;
        U[k][b] = sn[t] * ua + cs[t] * ub;
      }
      __syncthreads();
    }
  }
  if (tid == 0) {
    // descending eigenvalues above 1e-12 of the largest
    int ord[16];
    for (int i = 0; i < nb; ++i) ord[i] = i;
    for (int i = 1; i < nb; ++i)
      for (int j = i; j > 0 && A[ord[j]][ord[j]] > A[ord[j - 1]][ord[j - 1]]; --j) {
        const int t = ord[j]; ord[j] = ord[j - 1]; ord[j - 1] = t;
      }
    const double lmax = A[ord[0]][ord[0]];
    int r = 0;
    for (int i = 0; i < nb; ++i) {
      const double l = A[ord[i]][ord[i]];
      if (l > 1e-12 * lmax && l > 0) keep[r++] = ord[i];
    }
    rr = r;
    if (r < nb) *rank_short = 1;
  }
  __syncthreads();
  for (int x = tid; x < nb * nb; x += kSvqbThreads) {
    const int i = x % nb, q = x / nb;
    M[x] = q < rr ? d[i] * U[i][keep[q]] / sqrt(A[keep[q]][keep[q]]) : 0.0;
  }
}

// The dynamic shared-memory limits are set once per process to the largest size any launch uses,
// so concurrent contexts never race on them.
std::once_flag g_attr_once;
void set_attributes() {
  std::call_once(g_attr_once, [] {
    cudaFuncSetAttribute(k_rows<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)rows_smem<1>(kRowsMaxM));
    cudaFuncSetAttribute(k_rows<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)rows_smem<2>(kRowsMaxM));
    cudaFuncSetAttribute(k_rows<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)rows_smem<4>(kRowsMaxM4));
    cudaFuncSetAttribute(k_rows_gram<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)fuse_smem<1>(kFuseMaxM));
    cudaFuncSetAttribute(k_rows_gram<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)fuse_smem<2>(kFuseMaxM));
  });
}

}  // namespace

void svqb_factor(const double* S, int nb, double* M, int* rank_short, cudaStream_t s) {
  note_launch();
  k_svqb_factor<<<1, kSvqbThreads, 0, s>>>(S, nb, M, rank_short);
}

int64_t proj_gram_scratch(int M, int P) {
  // blocks x row groups x Mc <= kBlocks x kGramSlab for every slab width (groups x tiles <= 96)
  (void)M;
  return (int64_t)kBlocks * kGramSlab * P;
}

bool proj_gram(const double* A, int lda, const double* B, int ldb, int64_t n, int M, int P,
               double alpha, double beta, double* C, int ldc, double* part, cudaStream_t s) {
  if (M <= 0 || P <= 0) return true;
  if (P > 16 || lda < M || ldb < P) return false;
  int nblk = kBlocks;
  if (n < (int64_t)nblk * 64) nblk = (int)std::max<int64_t>(1, (n + 63) / 64);
  for (int a0 = 0; a0 < M; a0 += kGramSlab) {
    const int Mc = std::min(kGramSlab, M - a0);
    // up to 16 tiles of C: 16 warps, one tile each, eight k-steps in flight; up to 64 tiles: 32
    // warps, two tiles each, four k-steps; wider: 16 warps, six tiles each, two k-steps (measured
    // on 380k rows, P = 16: 0.39 ms against 0.47 ms at M = 512 for the middle form, and 0.50
    // against 0.55 ms at M = 672 for the wide one)
    const int form = Mc <= 8 * kGramWarps ? 0 : (Mc <= 8 * 2 * 32 ? 1 : 2);
    const int nparts = nblk * (form == 0   ? gram_groups(Mc, 1, kGramWarps)
                               : form == 1 ? gram_groups(Mc, 2, 32)
                                           : gram_groups(Mc, kGramTiles, kGramWarps));
    note_launch();
    if (form == 0) {
      if (P <= 8) k_gram<1, 1, 8, kGramWarps><<<nblk, kGramThreads, 0, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
      else k_gram<2, 1, 8, kGramWarps><<<nblk, kGramThreads, 0, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
    } else if (form == 1) {
      if (P <= 8) k_gram<1, 2, 4, 32><<<nblk, 1024, 0, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
      else k_gram<2, 2, 4, 32><<<nblk, 1024, 0, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
    } else {
      if (P <= 8)
        k_gram<1, kGramTiles, kGramUnroll, kGramWarps><<<nblk, kGramThreads, 0, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
      else
        k_gram<2, kGramTiles, kGramUnroll, kGramWarps><<<nblk, kGramThreads, 0, s>>>(A + a0, lda, B, ldb, n, Mc, P, part);
    }
    note_launch();
    k_gram_reduce<<<(Mc * P + 31) / 32, kRedWarps * 32, 0, s>>>(part, nparts, Mc, P, alpha, beta,
                                                                 C + a0, ldc);
  }
  return true;
}

bool proj_rows_gram(const double* A, int lda, const double* S1, int lds, double* W, int ldw,
                    int64_t n, int M, int P, double* C, int ldc, double* part, cudaStream_t s) {
  if (M <= 0 || P <= 0 || n <= 0) return true;
  if (M > kFuseMaxM || P > 16 || lda < M || ldw < P) return false;
  set_attributes();
  int nblk = kBlocks;
  if (n < (int64_t)nblk * kFuseChunk)
    nblk = (int)std::max<int64_t>(1, (n + kFuseChunk - 1) / kFuseChunk);
  note_launch();
  if (P <= 8)
    k_rows_gram<1><<<nblk, kThreads, fuse_smem<1>(M), s>>>(A, lda, S1, lds, W, ldw, n, M, P, part);
  else
    k_rows_gram<2><<<nblk, kThreads, fuse_smem<2>(M), s>>>(A, lda, S1, lds, W, ldw, n, M, P, part);
  note_launch();
  k_gram_reduce<<<(M * P + 31) / 32, kRedWarps * 32, 0, s>>>(part, nblk, M, P, 1.0, 0.0, C, ldc);
  return true;
}

void proj_rows(const double* A, int lda, const double* S, int lds, int64_t n, int M, int P,
               double alpha, double beta, double* Out, int ldo, cudaStream_t s) {
  if (n <= 0 || P <= 0) return;
  set_attributes();
  const int64_t tiles = (n + 7) / 8;
  const int g = (int)std::min<int64_t>(kBlocks, (tiles + 31) / 32);
  // 32-column slabs when S's rows fit beside them in shared memory: half the passes over A
  const int cw = (P > 16 && M <= kRowsMaxM4) ? 32 : 16;
  for (int c0 = 0; c0 < P; c0 += cw) {
    const int pc = std::min(cw, P - c0);
    double* Oc = Out + c0;
    // slabs of S rows; every slab after the first adds into Out
    for (int a0 = 0; a0 < std::max(M, 1); a0 += kRowsMaxM) {
      const int Mc = std::min(kRowsMaxM, M - a0);
      const double* Sc = S + (int64_t)c0 * lds + a0;
      const double bt = a0 == 0 ? beta : 1.0;
      note_launch();
      if (pc > 16)
        k_rows<4><<<g, kThreads, rows_smem<4>(std::max(Mc, 1)), s>>>(A + a0, lda, Sc, lds, n,
                                                                     Mc, pc, alpha, bt, Oc, ldo);
      else if (pc <= 8)
        k_rows<1><<<g, kThreads, rows_smem<1>(std::max(Mc, 1)), s>>>(A + a0, lda, Sc, lds, n,
                                                                     Mc, pc, alpha, bt, Oc, ldo);
      else
        k_rows<2><<<g, kThreads, rows_smem<2>(std::max(Mc, 1)), s>>>(A + a0, lda, Sc, lds, n,
                                                                     Mc, pc, alpha, bt, Oc, ldo);
    }
  }
}

}  // namespace vhci
