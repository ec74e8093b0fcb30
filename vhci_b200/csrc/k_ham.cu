// Hamiltonian kernels: the connection-driven sparse build (replacing the reference's O(N^2) pair
// loop, Ham.cpp:228-326), the SpMM that drives the eigensolver, and the Davidson vector helpers.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <string>

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

}  // namespace

namespace {

// One warp per row; lanes stride over the connection groups, probe the basis hash and compact
// the hits with a ballot, so a row's entries land in group order (deterministic layout).  Rows
// row0 .. row0 + n - 1 of the basis are built (all of them, or one rank's block of a sharded
// matrix); rowcnt, rowptr and diag are indexed from row0, columns are basis indices.
template <int W, bool FILL>
__global__ void __launch_bounds__(256) k_hbuild(const uint64_t* __restrict__ keys, int64_t row0,
                                                int64_t n, KeyLayout L, HashView basis, ConnDev cd,
                                                int32_t* __restrict__ rowcnt,
                                                const int64_t* __restrict__ rowptr,
                                                int32_t* __restrict__ col,
                                                double* __restrict__ val,
                                                float* __restrict__ valf,
                                                double* __restrict__ diag) {
  __shared__ uint32_t s_binom[kBinomElems];
  __shared__ uint8_t s_exc[8][128];
  fill_binom(s_binom);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
       i += warps) {
    uint64_t k[W];
    load_key<W>(keys, row0 + i, k);
    const int64_t pos = FILL ? rowptr[i] : 0;
    int cnt = 0;
    for_each_group<W>(cd, k, L, s_exc[threadIdx.x >> 5], s_binom, [&](int64_t u) {
      int64_t j = -1;
      GroupDev g;
      if (u >= 0) {
        g = cd.groups[u];
        uint64_t t[W];
        if (group_target<W>(cd, u, g, k, L, t)) j = hash_find<W>(basis, t, key_hash<W>(t));
      }
      const unsigned b = __ballot_sync(0xffffffffu, j >= 0);
      if (FILL && j >= 0) {
        const int64_t p = pos + cnt + __popc(b & lanemask_lt());
        col[p] = (int32_t)j;
        const double v = group_value<W>(cd, g.tb, g.te, k, L);
        if (valf) valf[p] = (float)v; else val[p] = v;
      }
      cnt += __popc(b);
    });
    if (lane == 0) {
      if (FILL) diag[i] = diag_value<W>(cd, k, L);
      else rowcnt[i] = cnt;
    }
  }
}

template <int W>
void hbuild_count_launch(const uint64_t* keys, int64_t row0, int64_t n, KeyLayout L,
                         HashView basis, ConnDev cd, int32_t* rowcnt, cudaStream_t s) {
  note_launch(); k_hbuild<W, false><<<grid_for(n * 32, 256, 148 * 8), 256, 0, s>>>(
      keys, row0, n, L, basis, cd, rowcnt, nullptr, nullptr, nullptr, nullptr, nullptr);
}
template <int W>
void hbuild_fill_launch(const uint64_t* keys, int64_t row0, int64_t n, KeyLayout L,
                        HashView basis, ConnDev cd, const int64_t* rowptr, int32_t* col,
                        double* val, float* valf, double* diag, cudaStream_t s) {
  note_launch(); k_hbuild<W, true><<<grid_for(n * 32, 256, 148 * 8), 256, 0, s>>>(
      keys, row0, n, L, basis, cd, nullptr, rowptr, col, val, valf, diag);
}

// Row-group SpMM, Y[:, 0:bp] = (D + H_off) X[:, 0:bp] for bp <= BP columns: a warp holds
// G = 32/BP rows, each handled by a group of BP lanes that own one column each and walk the row's
// entries together (the entry loads are broadcasts within the group and L1 hits across
// consecutive entries), eight entries per iteration so each lane keeps eight vector-row gathers in
// flight.  Entry loads are 16-byte (four columns, two or four values) after a scalar prologue to
// 4-entry alignment.  The diagonal term reads X row xrow0 + i (a rank's row block of a sharded
// matrix multiplies the gathered whole block); accum != 0 adds into Y instead (a later column
// panel).
template <int BP, typename VT>
__global__ void __launch_bounds__(256) k_spmm_rows(int64_t n, const int64_t* __restrict__ rowptr,
                                                   const int32_t* __restrict__ col,
                                                   const VT* __restrict__ val,
                                                   const double* __restrict__ diag,
                                                   const double* __restrict__ X, int ldx, int bp,
                                                   double* __restrict__ Y, int ldy, int accum,
                                                   int64_t xrow0) {
  constexpr int G = 32 / BP;
  const int lane = threadIdx.x & 31;
  const int grp = lane / BP, cc = lane % BP;
  const bool active = cc < bp;
  const int64_t stride = (int64_t)gridDim.x * (blockDim.x >> 5) * G;
  for (int64_t i = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * G + grp;
       i < n; i += stride) {
    const int64_t beg = __ldg(rowptr + i), end = __ldg(rowptr + i + 1);
    double acc = 0.0;
    if (active && (!accum || end > beg)) {
      auto gx = [&](int j) { return __ldg(X + (int64_t)j * ldx + cc); };
      int64_t e = beg;
      for (; e < end && (e & 3); ++e) acc = fma((double)__ldg(val + e), gx(__ldg(col + e)), acc);
      for (; e + 8 <= end; e += 8) {
        const int4 ja = __ldg(reinterpret_cast<const int4*>(col + e));
        const int4 jb = __ldg(reinterpret_cast<const int4*>(col + e + 4));
        double v[8];
        if constexpr (sizeof(VT) == 8) {
          const double2 v01 = __ldg(reinterpret_cast<const double2*>(val + e));
          const double2 v23 = __ldg(reinterpret_cast<const double2*>(val + e + 2));
          const double2 v45 = __ldg(reinterpret_cast<const double2*>(val + e + 4));
          const double2 v67 = __ldg(reinterpret_cast<const double2*>(val + e + 6));
          v[0] = v01.x; v[1] = v01.y; v[2] = v23.x; v[3] = v23.y;
          v[4] = v45.x; v[5] = v45.y; v[6] = v67.x; v[7] = v67.y;
        } else {
          const float4 va = __ldg(reinterpret_cast<const float4*>(val + e));
          const float4 vb = __ldg(reinterpret_cast<const float4*>(val + e + 4));
          v[0] = va.x; v[1] = va.y; v[2] = va.z; v[3] = va.w;
          v[4] = vb.x; v[5] = vb.y; v[6] = vb.z; v[7] = vb.w;
        }
        const double x0 = gx(ja.x), x1 = gx(ja.y), x2 = gx(ja.z), x3 = gx(ja.w);
        const double x4 = gx(jb.x), x5 = gx(jb.y), x6 = gx(jb.z), x7 = gx(jb.w);
        acc = fma(v[0], x0, acc);
        acc = fma(v[1], x1, acc);
        acc = fma(v[2], x2, acc);
        acc = fma(v[3], x3, acc);
        acc = fma(v[4], x4, acc);
        acc = fma(v[5], x5, acc);
        acc = fma(v[6], x6, acc);
        acc = fma(v[7], x7, acc);
      }
#pragma unroll 4
      for (; e < end; ++e) acc = fma((double)__ldg(val + e), gx(__ldg(col + e)), acc);
      if (accum) Y[i * ldy + cc] += acc;
      else Y[i * ldy + cc] = fma(diag[i], X[(xrow0 + i) * ldx + cc], acc);
    }
  }
}

// Column-pair form of the row-group SpMM: each lane owns two adjacent columns and gathers them as
// one 16-byte load, so a 16-column block row (128 bytes) takes 8 lanes and a warp holds 4 rows;
// sixteen entries per iteration keep sixteen 16-byte gathers in flight per lane.  The product is
// bound by the latency of those gathers (L2 at under half its throughput), so the register budget
// is set for four resident blocks per SM (64 registers): the compiler then keeps all sixteen
// gathers in flight, where at its own choice (40 registers, six blocks) it kept fewer.  Measured on
// the 380k-state workload-1 matrix (b = 16): 2.62 ms, against 2.96 ms at 40 registers and 3.35 ms
// for one column per lane.  Needs X and Y 16-byte aligned with even strides (the launcher checks).
template <int BQ, typename VT>
__global__ void __launch_bounds__(256, 4) k_spmm_pairs(int64_t n, const int64_t* __restrict__ rowptr,
                                                    const int32_t* __restrict__ col,
                                                    const VT* __restrict__ val,
                                                    const double* __restrict__ diag,
                                                    const double* __restrict__ X, int ldx, int bq,
                                                    double* __restrict__ Y, int ldy, int accum,
                                                    int64_t xrow0) {
  constexpr int G = 32 / BQ, U = 16;
  const int lane = threadIdx.x & 31;
  const int grp = lane / BQ, cc = lane % BQ;
  const bool active = cc < bq;
  const double2* __restrict__ X2 = reinterpret_cast<const double2*>(X);
  const int ldx2 = ldx >> 1, ldy2 = ldy >> 1;
  const int64_t stride = (int64_t)gridDim.x * (blockDim.x >> 5) * G;
  for (int64_t i = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * G + grp;
       i < n; i += stride) {
    const int64_t beg = __ldg(rowptr + i), end = __ldg(rowptr + i + 1);
    if (!active || (accum && end == beg)) continue;
    double ax = 0.0, ay = 0.0;
    auto gx = [&](int j) { return __ldg(X2 + (int64_t)j * ldx2 + cc); };
    int64_t e = beg;
    for (; e < end && (e & 3); ++e) {
      const double v = (double)__ldg(val + e);
      const double2 x = gx(__ldg(col + e));
      ax = fma(v, x.x, ax);
      ay = fma(v, x.y, ay);
    }
    for (; e + U <= end; e += U) {
      int j[U];
      double v[U];
#pragma unroll
      for (int u = 0; u < U; u += 4) {
        const int4 jj = __ldg(reinterpret_cast<const int4*>(col + e + u));
        j[u] = jj.x; j[u + 1] = jj.y; j[u + 2] = jj.z; j[u + 3] = jj.w;
        if constexpr (sizeof(VT) == 8) {
          const double2 va = __ldg(reinterpret_cast<const double2*>(val + e + u));
          const double2 vb = __ldg(reinterpret_cast<const double2*>(val + e + u + 2));
          v[u] = va.x; v[u + 1] = va.y; v[u + 2] = vb.x; v[u + 3] = vb.y;
        } else {
          const float4 vf = __ldg(reinterpret_cast<const float4*>(val + e + u));
          v[u] = vf.x; v[u + 1] = vf.y; v[u + 2] = vf.z; v[u + 3] = vf.w;
        }
      }
      double2 x[U];
#pragma unroll
      for (int u = 0; u < U; ++u) x[u] = gx(j[u]);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        ax = fma(v[u], x[u].x, ax);
        ay = fma(v[u], x[u].y, ay);
      }
    }
#pragma unroll 4
    for (; e < end; ++e) {
      const double v = (double)__ldg(val + e);
      const double2 x = gx(__ldg(col + e));
      ax = fma(v, x.x, ax);
      ay = fma(v, x.y, ay);
    }
    double2* y = reinterpret_cast<double2*>(Y) + i * ldy2 + cc;
    if (accum) {
      const double2 o = *y;
      *y = make_double2(o.x + ax, o.y + ay);
    } else {
      const double d = diag[i];
      const double2 xi = X2[(xrow0 + i) * ldx2 + cc];
      *y = make_double2(fma(d, xi.x, ax), fma(d, xi.y, ay));
    }
  }
}

// Mixed-precision form: the gathered vector block is FP32 (each lane owns four adjacent columns,
// one 16-byte float4 gather), the matrix values FP32, the accumulation FP64, and the diagonal term
// multiplies the FP64 block Xd (row i of the rows held, stride ldd).  A 16-column FP32 block row
// is 64 bytes, half the gathered bytes of the FP64 form.  Register budget as for k_spmm_pairs.
template <int BQ>
__global__ void __launch_bounds__(256, 4) k_spmm_f32x(int64_t n, const int64_t* __restrict__ rowptr,
                                                   const int32_t* __restrict__ col,
                                                   const float* __restrict__ val,
                                                   const double* __restrict__ diag,
                                                   const float* __restrict__ X, int ldx, int bq,
                                                   const double* __restrict__ Xd, int ldd,
                                                   double* __restrict__ Y, int ldy) {
  constexpr int G = 32 / BQ, U = 16;
  const int lane = threadIdx.x & 31;
  const int grp = lane / BQ, cc = lane % BQ;
  const bool active = cc < bq;
  const float4* __restrict__ X4 = reinterpret_cast<const float4*>(X);
  const int ldx4 = ldx >> 2;
  const int64_t stride = (int64_t)gridDim.x * (blockDim.x >> 5) * G;
  for (int64_t i = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * G + grp;
       i < n; i += stride) {
    if (!active) continue;
    const int64_t beg = __ldg(rowptr + i), end = __ldg(rowptr + i + 1);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    auto acc = [&](double v, float4 x) {
      a0 = fma(v, (double)x.x, a0);
      a1 = fma(v, (double)x.y, a1);
      a2 = fma(v, (double)x.z, a2);
      a3 = fma(v, (double)x.w, a3);
    };
    auto gx = [&](int j) { return __ldg(X4 + (int64_t)j * ldx4 + cc); };
    int64_t e = beg;
    for (; e < end && (e & 3); ++e) acc((double)__ldg(val + e), gx(__ldg(col + e)));
    for (; e + U <= end; e += U) {
      int j[U];
      float v[U];
#pragma unroll
      for (int u = 0; u < U; u += 4) {
        const int4 jj = __ldg(reinterpret_cast<const int4*>(col + e + u));
        j[u] = jj.x; j[u + 1] = jj.y; j[u + 2] = jj.z; j[u + 3] = jj.w;
        const float4 vf = __ldg(reinterpret_cast<const float4*>(val + e + u));
        v[u] = vf.x; v[u + 1] = vf.y; v[u + 2] = vf.z; v[u + 3] = vf.w;
      }
      float4 x[U];
#pragma unroll
      for (int u = 0; u < U; ++u) x[u] = gx(j[u]);
#pragma unroll
      for (int u = 0; u < U; ++u) acc((double)v[u], x[u]);
    }
#pragma unroll 4
    for (; e < end; ++e) acc((double)__ldg(val + e), gx(__ldg(col + e)));
    const double d = diag[i];
    const double* xd = Xd + i * ldd + 4 * cc;
    double* y = Y + i * ldy + 4 * cc;
    y[0] = fma(d, xd[0], a0);
    y[1] = fma(d, xd[1], a1);
    y[2] = fma(d, xd[2], a2);
    y[3] = fma(d, xd[3], a3);
  }
}

template <typename VT>
void spmm_rows_launch(int64_t n, const int64_t* rowptr, const int32_t* col, const VT* val,
                      const double* diag, const double* X, int ldx, int b, double* Y, int ldy,
                      int accum, int64_t xrow0, cudaStream_t s) {
  const bool pairs = (b % 2 == 0) && (ldx % 2 == 0) && (ldy % 2 == 0) &&
                     (reinterpret_cast<uintptr_t>(X) % 16 == 0) &&
                     (reinterpret_cast<uintptr_t>(Y) % 16 == 0);
  if (pairs) {
    const int BQ = b <= 8 ? 4 : (b <= 16 ? 8 : 16);  // lanes per row; columns per launch 2 BQ
    const int gr = grid_for(n * BQ, 256, 148 * 16);
    for (int c0 = 0; c0 < b; c0 += 2 * BQ) {
      const int bq = std::min(BQ, (b - c0) / 2);
      note_launch();
      if (BQ == 16)
        k_spmm_pairs<16, VT><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bq, Y + c0, ldy, accum, xrow0);
      else if (BQ == 8)
        k_spmm_pairs<8, VT><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bq, Y + c0, ldy, accum, xrow0);
      else
        k_spmm_pairs<4, VT><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bq, Y + c0, ldy, accum, xrow0);
    }
    return;
  }
  const int BP = b <= 8 ? 8 : (b <= 16 ? 16 : 32);
  const int gr = grid_for(n * BP, 256, 148 * 16);
  for (int c0 = 0; c0 < b; c0 += BP) {
    const int bp = std::min(BP, b - c0);
    note_launch();
    if (BP == 32)
      k_spmm_rows<32, VT><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bp, Y + c0, ldy, accum, xrow0);
    else if (BP == 16)
      k_spmm_rows<16, VT><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bp, Y + c0, ldy, accum, xrow0);
    else
      k_spmm_rows<8, VT><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bp, Y + c0, ldy, accum, xrow0);
  }
}

__global__ void k_resid_part(const double* __restrict__ X, const double* __restrict__ HX, int64_t n,
                             int ld, int kk, const double* __restrict__ theta,
                             double* __restrict__ part) {
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = blockIdx.x * per, hi = min(n, lo + per);
  for (int c = threadIdx.x; c < kk; c += blockDim.x) {
    const double th = theta[c];
    double s = 0.0;
    for (int64_t i = lo; i < hi; ++i) {
      const double r = HX[i * ld + c] - th * X[i * ld + c];
      s = fma(r, r, s);
    }
    part[(int64_t)blockIdx.x * kk + c] = s;
  }
}

__global__ void k_sum_parts(const double* __restrict__ part, int nblk, int kk,
                            double* __restrict__ out, int accumulate) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kk; c += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * kk + c];
    out[c] = accumulate ? out[c] + s : s;
  }
}

__global__ void k_copy_cols(const double* __restrict__ src, int lds, double* __restrict__ dst,
                            int ldd, int64_t n, int ncol) {
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n * ncol;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / ncol;
    const int c = (int)(idx % ncol);
    dst[i * ldd + c] = src[i * lds + c];
  }
}

template <typename VT>
__global__ void k_dense_from_csr(int64_t n, const int64_t* __restrict__ rowptr,
                                 const int32_t* __restrict__ col, const VT* __restrict__ val,
                                 const double* __restrict__ diag, double* __restrict__ A) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) A[i * n + col[e]] = (double)val[e];
    A[i * n + i] = diag[i];
  }
}

__global__ void k_fill_zero(double* p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = 0.0;
}

}  // namespace

void hbuild_count(const uint64_t* keys, int64_t row0, int64_t n, KeyLayout L, HashView basis,
                  ConnDev cd, int32_t* rowcnt, cudaStream_t s) {
  if (n <= 0) return;
  VHCI_DISPATCH_W(L.W, hbuild_count_launch, keys, row0, n, L, basis, cd, rowcnt, s);
}

void hbuild_fill(const uint64_t* keys, int64_t row0, int64_t n, KeyLayout L, HashView basis,
                 ConnDev cd, const int64_t* rowptr, int32_t* col, double* val, float* valf,
                 double* diag, cudaStream_t s) {
  if (n <= 0) return;
  VHCI_DISPATCH_W(L.W, hbuild_fill_launch, keys, row0, n, L, basis, cd, rowptr, col, val, valf,
                  diag, s);
}

// ---- column panels: the off-diagonal entries regrouped by column range -----------------------
// When the gathered block no longer fits in L2, the product runs once per column panel, so the
// rows gathered in one pass (one panel of the block) stay L2-resident while H streams once.
// Layout: entries of panel p for row i at [prow[p n + i], prow[p n + i + 1]); within a (panel,
// row) cell entries keep their CSR order, so the product is deterministic.

namespace {

// cnt[p n + i] = entries of row i in column panel p (cnt zeroed by the caller).
__global__ void __launch_bounds__(256) k_panel_count(int64_t n, const int64_t* __restrict__ rowptr,
                                                     const int32_t* __restrict__ col, int64_t cw,
                                                     int32_t* __restrict__ cnt) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
       i += warps) {
    const int64_t beg = rowptr[i], end = rowptr[i + 1];
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
      const int64_t e = e0 + lane;
      const bool v = e < end;
      const int p = v ? (int)(col[e] / cw) : -1;
      const unsigned peers = __match_any_sync(full, p);
      if (v && (peers & lanemask_lt()) == 0) atomicAdd(cnt + (int64_t)p * n + i, __popc(peers));
    }
  }
}

template <typename VT>
__global__ void __launch_bounds__(256) k_panel_fill(int64_t n, const int64_t* __restrict__ rowptr,
                                                    const int32_t* __restrict__ col,
                                                    const VT* __restrict__ val, int64_t cw, int P,
                                                    const int64_t* __restrict__ prow,
                                                    int32_t* __restrict__ pcol,
                                                    VT* __restrict__ pval) {
  __shared__ int s_run[8][kMaxPanels];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int* run = s_run[threadIdx.x >> 5];
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
       i += warps) {
    for (int p = lane; p < P; p += 32) run[p] = 0;
    __syncwarp();
    const int64_t beg = rowptr[i], end = rowptr[i + 1];
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
      const int64_t e = e0 + lane;
      const bool v = e < end;
      const int p = v ? (int)(col[e] / cw) : -1;
      const unsigned peers = __match_any_sync(full, p);
      const unsigned below = peers & lanemask_lt();
      if (v) {
        const int64_t pos = prow[(int64_t)p * n + i] + run[p] + __popc(below);
        pcol[pos] = col[e];
        pval[pos] = val[e];
      }
      __syncwarp();
      if (v && below == 0) run[p] += __popc(peers);
      __syncwarp();
    }
  }
}

}  // namespace

void panel_count(int64_t n, const int64_t* rowptr, const int32_t* col, int64_t cw, int32_t* cnt,
                 cudaStream_t s) {
  if (n <= 0) return;
  note_launch(); k_panel_count<<<grid_for(n * 32, 256, 148 * 8), 256, 0, s>>>(n, rowptr, col, cw, cnt);
}

void panel_fill(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val,
                const float* valf, int64_t cw, int P, const int64_t* prow, int32_t* pcol,
                double* pval, float* pvalf, cudaStream_t s) {
  if (n <= 0) return;
  const int g = grid_for(n * 32, 256, 148 * 8);
  note_launch();
  if (valf) k_panel_fill<float><<<g, 256, 0, s>>>(n, rowptr, col, valf, cw, P, prow, pcol, pvalf);
  else k_panel_fill<double><<<g, 256, 0, s>>>(n, rowptr, col, val, cw, P, prow, pcol, pval);
}

void spmm_panels(int64_t n, int P, const int64_t* prow, const int32_t* pcol, const double* pval,
                 const float* pvalf, const double* diag, const double* X, int ldx, int b,
                 double* Y, int ldy, int64_t xrow0, cudaStream_t s) {
  if (n <= 0 || b <= 0) return;
  for (int p = 0; p < P; ++p) {
    if (pvalf) spmm_rows_launch<float>(n, prow + (int64_t)p * n, pcol, pvalf, diag, X, ldx, b, Y, ldy, p > 0, xrow0, s);
    else spmm_rows_launch<double>(n, prow + (int64_t)p * n, pcol, pval, diag, X, ldx, b, Y, ldy, p > 0, xrow0, s);
  }
}

bool spmm_f32x(int64_t n, const int64_t* rowptr, const int32_t* col, const float* val,
               const double* diag, const float* X, int ldx, int b, const double* Xd, int ldd,
               double* Y, int ldy, cudaStream_t s) {
  if (n <= 0 || b <= 0) return true;
  if (b % 4 || ldx % 4 || reinterpret_cast<uintptr_t>(X) % 16) return false;
  const int BQ = b <= 16 ? 4 : 8;  // lanes per row; 4 BQ columns per launch
  const int gr = grid_for(n * BQ, 256, 148 * 16);
  for (int c0 = 0; c0 < b; c0 += 4 * BQ) {
    const int bq = std::min(BQ, (b - c0) / 4);
    note_launch();
    if (BQ == 8)
      k_spmm_f32x<8><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bq, Xd + c0, ldd, Y + c0, ldy);
    else
      k_spmm_f32x<4><<<gr, 256, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bq, Xd + c0, ldd, Y + c0, ldy);
  }
  return true;
}

// Compact FP32 copy of ncol columns of a row-major FP64 block (rounded to nearest).
__global__ void k_copy_cols_f32(const double* __restrict__ src, int lds, float* __restrict__ dst,
                                int ldd, int64_t n, int ncol) {
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n * ncol;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / ncol;
    const int c = (int)(idx % ncol);
    dst[i * ldd + c] = (float)src[i * lds + c];
  }
}

void copy_cols_f32(const double* src, int lds, float* dst, int ldd, int64_t n, int ncol,
                   cudaStream_t s) {
  if (n <= 0 || ncol <= 0) return;
  note_launch();
  k_copy_cols_f32<<<grid_for(n * ncol, 256), 256, 0, s>>>(src, lds, dst, ldd, n, ncol);
}

void spmm(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val,
          const float* valf, const double* diag, const double* X, int ldx, int b, double* Y,
          int ldy, int64_t xrow0, cudaStream_t s) {
  if (n <= 0 || b <= 0) return;
  if (valf) spmm_rows_launch<float>(n, rowptr, col, valf, diag, X, ldx, b, Y, ldy, 0, xrow0, s);
  else spmm_rows_launch<double>(n, rowptr, col, val, diag, X, ldx, b, Y, ldy, 0, xrow0, s);
}

int residual_blocks(int64_t n) {
  int64_t b = (n + 1023) / 1024;
  if (b > 148 * 4) b = 148 * 4;
  if (b < 1) b = 1;
  return (int)b;
}

void residual_norms(const double* X, const double* HX, int64_t n, int ld, int kk,
                    const double* theta, double* part, int nblk, double* rn2, cudaStream_t s) {
  note_launch(); k_resid_part<<<nblk, 256, 0, s>>>(X, HX, n, ld, kk, theta, part);
  note_launch(); k_sum_parts<<<(kk + 255) / 256, 256, 0, s>>>(part, nblk, kk, rn2, 0);
}

void copy_cols(const double* src, int lds, double* dst, int ldd, int64_t n, int ncol,
               cudaStream_t s) {
  if (n <= 0 || ncol <= 0) return;
  note_launch(); k_copy_cols<<<grid_for(n * ncol, 256), 256, 0, s>>>(src, lds, dst, ldd, n, ncol);
}

void dense_from_csr(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val,
                    const float* valf, const double* diag, double* A, cudaStream_t s) {
  fill_zero(A, n * n, s);
  if (valf) { note_launch(); k_dense_from_csr<float><<<grid_for(n, 128), 128, 0, s>>>(n, rowptr, col, valf, diag, A); }
  else { note_launch(); k_dense_from_csr<double><<<grid_for(n, 128), 128, 0, s>>>(n, rowptr, col, val, diag, A); }
}

void fill_zero(double* p, int64_t n, cudaStream_t s) {
  if (n > 0) { note_launch(); k_fill_zero<<<grid_for(n, 256), 256, 0, s>>>(p, n); }
}

void reduce_parts(const double* part, int nblk, int nopt, double* out_accum, cudaStream_t s) {
  note_launch(); k_sum_parts<<<(nopt + 255) / 256, 256, 0, s>>>(part, nblk, nopt, out_accum, 1);
}

// ---- incremental build: the stored matrix of the first n_old states, extended by the rows of
// the states appended since (H is symmetric to the bit, so the new columns of the old rows are
// the new rows' entries transposed) ----
namespace {

// add[c] += 1 for every new-row entry in an old column c, and the transposed entries' keys
// (c << 32 | entry index) compacted through cnt (their order is fixed by the sort that follows)
__global__ void k_cross_keys(const int32_t* __restrict__ col, int64_t nnz, int64_t n_old,
                             int32_t* __restrict__ add, uint64_t* __restrict__ keys,
                             unsigned long long* __restrict__ cnt) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = col[e];
    if (c < n_old) {
      atomicAdd(add + c, 1);
      keys[atomicAdd(cnt, 1ull)] = ((uint64_t)(uint32_t)c << 32) | (uint64_t)e;
    }
  }
}

// entry -> row of the new rows' CSR (one warp per row)
__global__ void k_entry_rows(const int64_t* __restrict__ rp, int64_t nrows, int32_t* __restrict__ erow) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows;
       r += ((int64_t)gridDim.x * blockDim.x) >> 5)
    for (int64_t e = rp[r] + lane; e < rp[r + 1]; e += 32) erow[e] = (int32_t)r;
}

// merged row lengths: old rows keep their entries and gain add[i]; new rows as built
__global__ void k_merge_len(const int64_t* __restrict__ rp_old, const int32_t* __restrict__ add,
                            const int64_t* __restrict__ rp_new, int64_t n_old, int64_t nn,
                            int32_t* __restrict__ len) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_old + nn;
       i += (int64_t)gridDim.x * blockDim.x)
    len[i] = i < n_old ? (int32_t)(rp_old[i + 1] - rp_old[i]) + add[i]
                       : (int32_t)(rp_new[i - n_old + 1] - rp_new[i - n_old]);
}

// rows [rs[i], rs[i+1]) copied to rd[i].. (one warp per row)
template <typename VT>
__global__ void k_copy_rows(const int64_t* __restrict__ rs, const int32_t* __restrict__ cs,
                            const VT* __restrict__ vs, int64_t nrows, const int64_t* __restrict__ rd,
                            int32_t* __restrict__ cd, VT* __restrict__ vd) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows;
       r += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t b = rs[r], m = rs[r + 1] - b, d = rd[r];
    for (int64_t t = lane; t < m; t += 32) {
      cd[d + t] = cs[b + t];
      vd[d + t] = vs[b + t];
    }
  }
}

// the sorted transposed entries to the tails of the old rows: key t of column c goes to position
// rp_all[c] + (old length of c) + (t - first key of c), as column n_old + (its new row)
template <typename VT>
__global__ void k_cross_scatter(const uint64_t* __restrict__ keys, int64_t ncross,
                                const int64_t* __restrict__ xoff, const int64_t* __restrict__ rp_old,
                                const int64_t* __restrict__ rp_all, const int32_t* __restrict__ erow,
                                const VT* __restrict__ vnew, int64_t n_old, int32_t* __restrict__ cd,
                                VT* __restrict__ vd) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ncross;
       t += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[t];
    const int64_t c = (int64_t)(k >> 32), e = (int64_t)(k & 0xffffffffull);
    const int64_t pos = rp_all[c] + (rp_old[c + 1] - rp_old[c]) + (t - xoff[c]);
    cd[pos] = (int32_t)(n_old + erow[e]);
    vd[pos] = vnew[e];
  }
}

}  // namespace

void hmerge_cross_keys(const int32_t* col_new, int64_t nnz_new, int64_t n_old, int32_t* add,
                       uint64_t* keys, unsigned long long* cnt, cudaStream_t s) {
  if (nnz_new <= 0) return;
  note_launch();
  k_cross_keys<<<grid_for(nnz_new, 256, 148 * 8), 256, 0, s>>>(col_new, nnz_new, n_old, add, keys, cnt);
}

void hmerge_entry_rows(const int64_t* rp_new, int64_t nn, int32_t* erow, cudaStream_t s) {
  if (nn <= 0) return;
  note_launch();
  k_entry_rows<<<grid_for(nn * 32, 256, 148 * 8), 256, 0, s>>>(rp_new, nn, erow);
}

void hmerge_lengths(const int64_t* rp_old, const int32_t* add, const int64_t* rp_new, int64_t n_old,
                    int64_t nn, int32_t* len, cudaStream_t s) {
  note_launch();
  k_merge_len<<<grid_for(n_old + nn, 256, 148 * 8), 256, 0, s>>>(rp_old, add, rp_new, n_old, nn, len);
}

void hmerge_copy_rows(const int64_t* rs, const int32_t* cs, const double* vs, const float* vsf,
                      int64_t nrows, const int64_t* rd, int32_t* cd, double* vd, float* vdf,
                      cudaStream_t s) {
  if (nrows <= 0) return;
  note_launch();
  const int g = grid_for(nrows * 32, 256, 148 * 8);
  if (vsf) k_copy_rows<float><<<g, 256, 0, s>>>(rs, cs, vsf, nrows, rd, cd, vdf);
  else k_copy_rows<double><<<g, 256, 0, s>>>(rs, cs, vs, nrows, rd, cd, vd);
}

void hmerge_cross_scatter(const uint64_t* keys, int64_t ncross, const int64_t* xoff,
                          const int64_t* rp_old, const int64_t* rp_all, const int32_t* erow,
                          const double* vnew, const float* vnewf, int64_t n_old, int32_t* cd,
                          double* vd, float* vdf, cudaStream_t s) {
  if (ncross <= 0) return;
  note_launch();
  const int g = grid_for(ncross, 256, 148 * 8);
  if (vnewf)
    k_cross_scatter<float><<<g, 256, 0, s>>>(keys, ncross, xoff, rp_old, rp_all, erow, vnewf, n_old, cd, vdf);
  else
    k_cross_scatter<double><<<g, 256, 0, s>>>(keys, ncross, xoff, rp_old, rp_all, erow, vnew, n_old, cd, vd);
}

}  // namespace vhci
