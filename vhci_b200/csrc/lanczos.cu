// Block thick-restart Lanczos for the lowest eigenpairs of the sparse Hamiltonian — the same
// method family as the reference's eigensolver (implicitly restarted Lanczos, SparseDiagonalize,
// Ham.cpp:347-370), organised for the GPU:
//   * blocks of b = 16 vectors; the SpMM gathers from a compact n x b copy of the block and
//     streams the matrix from HBM once per block;
//   * full reorthogonalisation (classical Gram-Schmidt, two passes) with FP64 tensor-core
//     projections (k_proj.cu), and the projected matrix T = Q^T H Q formed explicitly from the
//     stored H Q blocks;
//   * Rayleigh-Ritz (cuSOLVER syevd on T) only when the subspace is full; the kk = k + guard
//     lowest Ritz vectors are kept (thick restart) together with the pending Lanczos block, so the
//     kept Ritz vectors' residuals lie in the new subspace (Krylov-Schur property);
//   * convergence: ||H x - theta x|| <= tol * max(eps^(2/3), |theta|) for the k wanted pairs,
//     evaluated with explicit residuals at each restart (tol 1e-10 in the reference);
//   * heat-bath iterations start from b random combinations of the previous Ritz vectors
//     (zero-extended over the new states);
//   * on a sharded context every rank holds one contiguous row block of the Krylov basis (the
//     rows of its Hamiltonian block): the vector block is all-gathered before each product, the
//     projections' partial sums are all-reduced, the projected eigenproblem is solved on rank 0
//     and broadcast, and the Ritz vectors are all-gathered at the end, so every rank holds them
//     whole for the heat-bath selection.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "internal.h"

namespace vhci {

namespace {

// Cyclic Jacobi eigensolver for a small symmetric matrix (column-major, n <= 64): eigenvalues
// ascending in w, eigenvectors in the columns of V.
void jacobi_eig(int n, std::vector<double> A, std::vector<double>& w, std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  auto a = [&](int i, int j) -> double& { return A[(size_t)j * n + i]; };
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        tot += a(i, j) * a(i, j);
        if (i != j) off += a(i, j) * a(i, j);
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a(p, q);
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = cs * akp - sn * akq;
          a(k, q) = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = cs * apk - sn * aqk;
          a(q, k) = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
          V[(size_t)p * n + k] = cs * vkp - sn * vkq;
          V[(size_t)q * n + k] = sn * vkp + cs * vkq;
        }
      }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
  std::vector<double> V2((size_t)n * n);
  w.resize(n);
  for (int j = 0; j < n; ++j) {
    w[j] = a(ord[j], ord[j]);
    for (int i = 0; i < n; ++i) V2[(size_t)j * n + i] = V[(size_t)ord[j] * n + i];
  }
  V.swap(V2);
}

struct LWork {
  DBuf<double> Q, HQ, T, Yw, theta, Xb, HXb, W, S, M, part, rn2, Xc, gpart, Xg, gtmp;
  DBuf<float> Xf, Xgf;  // FP32 copies of the vector block (mixed precision)
  DBuf<int> short_flag;   // set by the device SVQB when a block loses rank
  bool exact = false;   // mixed precision: products with FP64 gathers (the final sweep)
  void release(cudaStream_t s) {
    Q.release(s); HQ.release(s); T.release(s); Yw.release(s); theta.release(s); Xb.release(s);
    HXb.release(s); W.release(s); S.release(s); M.release(s); part.release(s); rn2.release(s);
    Xc.release(s); gpart.release(s); Xg.release(s); gtmp.release(s); Xf.release(s);
    Xgf.release(s); short_flag.release(s);
  }
};

// Projections over the basis rows, on the FP64 tensor pipe (k_proj.cu).
// C (M x P, column-major) = alpha A^T B + beta C, A n x M and B n x P row-major.  On a sharded
// context the n rows are this rank's block and the partial product is summed over the ranks
// (beta must be 0 there).
int gemm_gram(vhci_ctx* c, LWork& w, const double* A, int lda, const double* B, int ldb, int64_t n,
              int M, int P, double alpha, double beta, double* C, int ldc) {
  if (M <= 0 || P <= 0) return VHCI_OK;
  const bool sh = is_sharded(c);
  if (sh && beta != 0.0) return fail(c, VHCI_E_STATE, "accumulating projection on a sharded context");
  double* out = C;
  int ldo = ldc;
  if (sh) {
    VCK(w.gtmp.reserve((size_t)M * P, c->st));
    out = w.gtmp.p;
    ldo = M;
  }
  VCK(w.gpart.reserve((size_t)proj_gram_scratch(M, P), c->st));
  if (!proj_gram(A, lda, B, ldb, n, M, P, alpha, beta, out, ldo, w.gpart.p, c->st))
    return fail(c, VHCI_E_INPUT, "projection with more than 16 right-hand columns");
  if (sh) {
    VTRY(comm_sum(c, out, (int64_t)M * P));
    VCK(cudaMemcpy2DAsync(C, ldc * sizeof(double), out, M * sizeof(double), M * sizeof(double), P,
                          cudaMemcpyDeviceToDevice, c->st));
  }
  return VHCI_OK;
}

// Out (n x P row-major) = alpha A S + beta Out, A n x M row-major, S M x P column-major.
int gemm_rows(vhci_ctx* c, const double* A, int lda, const double* S, int lds, int64_t n, int M,
              int P, double alpha, double beta, double* Out, int ldo) {
  if (n <= 0 || P <= 0) return VHCI_OK;
  (void)c;
  proj_rows(A, lda, S, lds, n, M, P, alpha, beta, Out, ldo, c->st);
  return VHCI_OK;
}

// The second and third Gram-Schmidt passes: W <- W - Q S1, then C = Q^T W (M x P, column-major),
// fused into one pass over Q's rows when the shapes allow (k_proj.cu), else as two products.
int gemm_rows_gram(vhci_ctx* c, LWork& w, const double* Q, int ldq, const double* S1, int lds,
                   int64_t n, int M, int P, double* W, int ldw, double* C, int ldc) {
  const bool sh = is_sharded(c);
  double* out = C;
  int ldo = ldc;
  if (sh) {
    VCK(w.gtmp.reserve((size_t)M * P, c->st));
    out = w.gtmp.p;
    ldo = M;
  }
  VCK(w.gpart.reserve((size_t)proj_gram_scratch(M, P), c->st));
  if (proj_rows_gram(Q, ldq, S1, lds, W, ldw, n, M, P, out, ldo, w.gpart.p, c->st)) {
    if (sh) {
      VTRY(comm_sum(c, out, (int64_t)M * P));
      VCK(cudaMemcpy2DAsync(C, ldc * sizeof(double), out, M * sizeof(double),
                            M * sizeof(double), P, cudaMemcpyDeviceToDevice, c->st));
    }
    return VHCI_OK;
  }
  VTRY(gemm_rows(c, Q, ldq, S1, lds, n, M, P, -1.0, 1.0, W, ldw));
  return gemm_gram(c, w, Q, ldq, W, ldw, n, M, P, 1.0, 0.0, C, ldc);
}

int syevd_l(vhci_ctx* c, double* A, int m, int lda, double* w) {
  int lwork = 0;
  VBL(cusolverDnDsyevd_bufferSize(c->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, m, A,
                                  lda, w, &lwork));
  VCK(c->solver_work.reserve(std::max(lwork, 1), c->st));
  VCK(c->solver_info.reserve(1, c->st));
  VBL(cusolverDnDsyevd(c->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, m, A, lda, w,
                       c->solver_work.p, lwork, c->solver_info.p));
  int info = 0;
  VCK(d2h(c, &info, c->solver_info.p, sizeof(int)));
  VCK(cudaStreamSynchronize(c->st));
  if (info != 0) return fail(c, VHCI_E_NOT_CONVERGED, "projected eigensolve failed");
  return VHCI_OK;
}

// Orthonormalise the nb columns of (B, ld) into (out, ldo) by SVQB with the small Gram matrix
// decomposed on the host; directions below 1e-12 of the largest are dropped.  *r = rank.
int svqb_small(vhci_ctx* c, LWork& w, int64_t n, const double* B, int ld, int nb, double* out,
               int ldo, int* r) {
  *r = 0;
  if (nb <= 0) return VHCI_OK;
  VCK(w.S.reserve((size_t)nb * nb, c->st));
  VTRY(gemm_gram(c, w, B, ld, B, ld, (int)n, nb, nb, 1.0, 0.0, w.S.p, nb));
  std::vector<double> S((size_t)nb * nb);
  VCK(d2h(c, S.data(), w.S.p, S.size() * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  std::vector<double> d(nb);
  double dmax = 0.0;
  for (int i = 0; i < nb; ++i) dmax = std::max(dmax, S[(size_t)i * nb + i]);
  for (int i = 0; i < nb; ++i) {
    const double s = S[(size_t)i * nb + i];
    d[i] = (s > 1e-28 * dmax && s > 1e-300) ? 1.0 / std::sqrt(s) : 0.0;
  }
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) S[(size_t)j * nb + i] *= d[i] * d[j];
  std::vector<double> L, U;
  jacobi_eig(nb, S, L, U);
  const double lmax = L[nb - 1];
  std::vector<int> keep;
  for (int j = nb - 1; j >= 0; --j)
    if (L[j] > 1e-12 * lmax && L[j] > 0) keep.push_back(j);
  const int rr = (int)keep.size();
  if (rr == 0) return VHCI_OK;
  std::vector<double> Mh((size_t)nb * rr);
  for (int q = 0; q < rr; ++q) {
    const double s = 1.0 / std::sqrt(L[keep[q]]);
    for (int i = 0; i < nb; ++i) Mh[(size_t)q * nb + i] = d[i] * U[(size_t)keep[q] * nb + i] * s;
  }
  VCK(w.M.reserve(Mh.size(), c->st));
  VCK(h2d(c, w.M.p, Mh.data(), Mh.size() * sizeof(double)));
  VTRY(gemm_rows(c, B, ld, w.M.p, nb, (int)n, nb, rr, 1.0, 0.0, out, ldo));
  *r = rr;
  return VHCI_OK;
}

// svqb_small without the host round trip: the factor is formed on the device (svqb_factor) and
// the block is assumed to keep its full rank nb, so nothing waits for the result; a lost
// direction sets w.short_flag, which the caller reads at its next synchronisation.
int svqb_dev(vhci_ctx* c, LWork& w, int64_t n, const double* B, int ld, int nb, double* out,
             int ldo) {
  VCK(w.S.reserve((size_t)nb * nb, c->st));
  VTRY(gemm_gram(c, w, B, ld, B, ld, (int)n, nb, nb, 1.0, 0.0, w.S.p, nb));
  VCK(w.M.reserve((size_t)nb * nb, c->st));
  svqb_factor(w.S.p, nb, w.M.p, w.short_flag.p, c->st);
  return gemm_rows(c, B, ld, w.M.p, nb, (int)n, nb, nb, 1.0, 0.0, out, ldo);
}

// Y = H X for a block of the held rows: X is first copied to a compact rows x b buffer so the SpMM
// gathers from a small, L2-resident array instead of rows of the wide basis; on a sharded context
// the ranks' compact blocks (rblk rows each) are all-gathered into the whole vector block first.
int apply_h_l(vhci_ctx* c, LWork& w, const double* X, int ldx, int b, double* Y, int ldy) {
  EventPair ev_e0e1;
  VCK(ev_e0e1.create());
  cudaEvent_t e0 = ev_e0e1.a, e1 = ev_e0e1.b;
  const int64_t nl = c->nrow, rb = c->rblk;
  VCK(cudaEventRecord(e0, c->st));
  // mixed precision: FP32 block gathers, FP64 accumulation and diagonal term (needs 16-byte
  // gathers of four columns; other widths, the final sweep and column panels gather FP64)
  const bool f32x = c->o.precision == 1 && !w.exact && b % 4 == 0;
  if (f32x) {
    VCK(w.Xf.reserve((size_t)std::max(nl, rb) * b, c->st));
    copy_cols_f32(X, ldx, w.Xf.p, b, nl, b, c->st);
    const float* Xfull = w.Xf.p;
    if (is_sharded(c)) {
      if (nl < rb) VCK(cudaMemsetAsync(w.Xf.p + (size_t)nl * b, 0, (rb - nl) * b * sizeof(float), c->st));
      VCK(w.Xgf.reserve((size_t)c->comm.nranks * rb * b, c->st));
      VTRY(comm_gather(c, w.Xf.p, w.Xgf.p, rb * b * (int64_t)sizeof(float)));
      Xfull = w.Xgf.p;
    }
    if (!spmm_f32x(nl, c->rowptr.p, c->col.p, c->valf.p, c->diag.p, Xfull, b, b, X, ldx, Y, ldy,
                   c->st))
      return fail(c, VHCI_E_STATE, "FP32 product with an unaligned block");
  } else {
    VCK(w.Xc.reserve((size_t)std::max(nl, rb) * b, c->st));
    copy_cols(X, ldx, w.Xc.p, b, nl, b, c->st);
    const double* Xfull = w.Xc.p;
    if (is_sharded(c)) {
      if (nl < rb) fill_zero(w.Xc.p + (size_t)nl * b, (rb - nl) * (int64_t)b, c->st);
      VCK(w.Xg.reserve((size_t)c->comm.nranks * rb * b, c->st));
      VTRY(comm_gather(c, w.Xc.p, w.Xg.p, rb * b * (int64_t)sizeof(double)));
      Xfull = w.Xg.p;
    }
    spmm_h(c, Xfull, b, b, Y, ldy);
  }
  VCK(cudaEventRecord(e1, c->st));
  VCK(cudaEventSynchronize(e1));
  VCK(cudaGetLastError());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  c->stats.ms_spmm += ms;
  c->stats.spmm_calls += 1;
  c->stats.spmm_cols += b;
  const int64_t sval = c->o.precision == 1 ? 4 : 8;
  const int64_t sx = f32x ? 4 : 8;
  c->stats.spmm_gather_bytes += c->nnz * (int64_t)b * sx;
  c->stats.spmm_bytes += c->nnz * (sval + 4) + (nl + 1) * 8 + nl * 8 + nl * (int64_t)b * (sx + 8);
  return VHCI_OK;
}

// Mixed precision, after the FP32-gather eigensolve: one Rayleigh-Ritz over the nk Ritz vectors
// held in w.Xb (rows held, ld kk; the first keff are the wanted pairs) with FP64 products H V (FP32 values, FP64 gathers and
// arithmetic), so the Ritz values and vectors carry no FP32 rounding of the vectors.  The rotated
// vectors replace w.Xb, their products land in w.HXb (ld kk), their residual norms (squared) in
// w.rn2 and their values in th.  Q and HQ (ld >= nk), no longer needed, are the work space.
int fp64_sweep(vhci_ctx* c, LWork& w, int kk, int nk, int keff, int ld, std::vector<double>& th) {
  const int64_t nl = c->nrow;
  cudaStream_t s = c->st;
  w.exact = true;
  for (int j0 = 0; j0 < nk; j0 += 16) {
    const int bw = std::min(16, nk - j0);
    VTRY(apply_h_l(c, w, w.Xb.p + j0, kk, bw, w.HQ.p + j0, ld));
  }
  w.exact = false;
  // T = V^T H V, column chunks of 16
  for (int j0 = 0; j0 < nk; j0 += 16) {
    const int bw = std::min(16, nk - j0);
    VTRY(gemm_gram(c, w, w.Xb.p, kk, w.HQ.p + j0, ld, nl, nk, bw, 1.0, 0.0,
                   w.T.p + (size_t)j0 * ld, ld));
  }
  VCK(cudaMemcpy2DAsync(w.Yw.p, ld * sizeof(double), w.T.p, ld * sizeof(double),
                        nk * sizeof(double), nk, cudaMemcpyDeviceToDevice, s));
  VTRY(syevd_l(c, w.Yw.p, nk, ld, w.theta.p));
  VTRY(comm_bcast0(c, w.Yw.p, (int64_t)ld * nk));
  VTRY(comm_bcast0(c, w.theta.p, nk));
  VTRY(gemm_rows(c, w.Xb.p, kk, w.Yw.p, ld, nl, nk, nk, 1.0, 0.0, w.Q.p, ld));
  VTRY(gemm_rows(c, w.HQ.p, ld, w.Yw.p, ld, nl, nk, nk, 1.0, 0.0, w.HXb.p, kk));
  copy_cols(w.Q.p, ld, w.Xb.p, kk, nl, nk, s);
  residual_norms(w.Xb.p, w.HXb.p, nl, kk, nk, w.theta.p, w.part.p, residual_blocks(nl), w.rn2.p, s);
  VTRY(comm_sum(c, w.rn2.p, nk));
  th.resize(nk);
  VCK(d2h(c, th.data(), w.theta.p, nk * sizeof(double)));
  std::vector<double> rn(nk);
  VCK(d2h(c, rn.data(), w.rn2.p, nk * sizeof(double)));
  VCK(cudaStreamSynchronize(s));
  double rmax = 0.0;
  for (int j = 0; j < keff; ++j)  // the wanted pairs; the guard vectors need not converge
    rmax = std::max(rmax, std::sqrt(std::max(rn[j], 0.0)) / std::max(1.0, std::fabs(th[j])));
  c->stats.mixed_max_residual = std::max(c->stats.mixed_max_residual, rmax);
  return VHCI_OK;
}

// Start vectors of the cold start: standard normal values drawn from the global (row, column)
// index, so every rank draws the same values for its rows whatever the sharding.
void random_rows(int64_t r0, int64_t rows, int b, std::vector<double>& out) {
  out.resize((size_t)rows * b);
  for (int64_t i = 0; i < rows; ++i)
    for (int j = 0; j < b; ++j) {
      const uint64_t key = ((uint64_t)(r0 + i) << 6) ^ (uint64_t)j;
      const double u1 = ((mix64(2 * key + 0x9E3779B97F4A7C15ull) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      const double u2 = ((mix64(2 * key + 1 + 0x9E3779B97F4A7C15ull) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      out[(size_t)i * b + j] = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
}

// Hands the Ritz block (this rank's rows, ld kk) to the context as its whole vectors: swapped in
// on an unsharded context, all-gathered from the ranks' row blocks (rblk rows each; the buffer
// holds at least that many) on a sharded one.
int publish_ritz(vhci_ctx* c, DBuf<double>& Xb, int kk, int nk, const std::vector<double>& th) {
  if (!is_sharded(c)) {
    c->X.swap(Xb);
  } else {
    c->X.release(c->st);
    VCK(c->X.reserve((size_t)c->comm.nranks * c->rblk * kk, c->st));
    VTRY(comm_gather(c, Xb.p, c->X.p, c->rblk * kk * (int64_t)sizeof(double)));
  }
  c->ldx = kk;
  c->nvec = nk;
  c->x_rows = c->n;
  c->E.assign(th.begin(), th.begin() + nk);
  VCK(cudaStreamSynchronize(c->st));
  return VHCI_OK;
}

}  // namespace

// Block size.  The SpMM's cost per vector column falls with the block width (the per-entry matrix
// loads are shared by more columns) and so does the reorthogonalisation cost per column (one pass
// over the basis serves the whole block), while wider blocks need more products in total.  Measured
// on B200 over the workload-1 solve (39k..380k states, k = 200): 16 is best at every size
// (VHCI_LANCZOS_BLOCK overrides it).
int lanczos_block(int64_t n) {
  (void)n;
  if (const char* e = std::getenv("VHCI_LANCZOS_BLOCK")) return std::max(4, std::min(32, std::atoi(e)));
  return 16;
}

// Guard vectors kept beyond the k wanted pairs at a restart: 60 % of k (at least 8;
// VHCI_LANCZOS_GUARD=p sets p %).  With subspace 2 kk + 2 b this needed 17-32 % fewer block
// products than 10 % with 3 kk + 2 b on three workloads (k = 50, 128, 200): keeping more of the
// Krylov space across restarts pays more than expanding further between them.
static int lanczos_guard(int k) {
  int pct = 60;
  if (const char* e = std::getenv("VHCI_LANCZOS_GUARD")) pct = std::max(1, std::min(200, std::atoi(e)));
  return std::max(8, k * pct / 100);
}

// Working set of the block Lanczos over n states for subspace factor `span`, on a rank holding
// `rows` of them: Q and H Q (rows x ld), the Ritz block and its product (rows x kk), the expansion
// block and its compact copy (rows x b), and the gathered vector block (n x b), in doubles.
static double lanczos_bytes(int64_t n, int64_t rows, int k, int span, int b) {
  const int kk = (int)std::min<int64_t>(n, k + lanczos_guard(k));
  const int mmax = (int)std::min<int64_t>(n, (int64_t)span * kk + 2 * b);
  const int ld = (mmax + b + 15) / 16 * 16;
  return 8.0 * (double)rows * (2.0 * ld + 2.0 * kk + 2.0 * b) + (rows < n ? 8.0 * n * b : 0.0);
}

// Working set of the memory-lean variant: Q (n x ld, span 2), the expansion block, its product,
// the compact copy (n x b each), the rotation chunk, and the output Ritz block (n x kk).
static double lanczos_lean_bytes(int64_t n, int64_t rows, int k, int b, int span = 2) {
  const int kk = (int)std::min<int64_t>(n, k + lanczos_guard(k));
  const int mmax = (int)std::min<int64_t>(n, (int64_t)span * kk + 2 * b);
  const int ld = (mmax + b + 15) / 16 * 16;
  return 8.0 * (double)rows * (ld + 3.0 * b + kk) + (rows < n ? 8.0 * n * (b + kk) : 0.0) + 2.6e8;
}

// Smallest eigensolver working set on this rank (the lean variant over the rows it will hold).
double lanczos_min_bytes(vhci_ctx* c, int k) {
  int64_t rows = c->n;
  if (is_sharded(c) && !dense_path(c->n, k)) rows = (c->n + c->comm.nranks - 1) / c->comm.nranks;
  return lanczos_lean_bytes(c->n, rows, k, lanczos_block(c->n)) + 1e9;
}

int block_lanczos_lean(vhci_ctx* c, int k);

// Relative residual tolerance of the FP32-gather eigensolve in mixed precision.
constexpr double kMixedTol = 1e-7;

int block_lanczos_impl(vhci_ctx* c, int k, bool dev_svqb);

// The block orthonormalisation of each step runs on the device (no host round trip per step) when
// the basis is much larger than the subspace, where a block losing rank does not happen in
// practice; if one does, the eigensolve is redone with the host factorisation, which drops the
// lost directions.
int block_lanczos(vhci_ctx* c, int k) { return block_lanczos_impl(c, k, true); }

int block_lanczos_impl(vhci_ctx* c, int k, bool dev_svqb) {
  const int64_t n = c->n;
  // rows held by this rank (all n unless sharded)
  const int64_t nl = c->nrow, r0 = c->row0, rb = std::max(c->rblk, nl);
  cudaStream_t s = c->st;
  const int guard = lanczos_guard(k);
  const int kk = (int)std::min<int64_t>(n, k + guard);
  const int b = lanczos_block(n);
  // subspace size: 2 kk + 2 b (VHCI_LANCZOS_SPAN overrides the factor 2); a basis too large for
  // that working set in the free device memory runs the memory-lean variant
  int span = 2;
  const double avail = device_available(c);
  if (const char* e = std::getenv("VHCI_LANCZOS_LEAN"))
    if (std::atoi(e) == 1) return block_lanczos_lean(c, k);
  if (const char* e = std::getenv("VHCI_LANCZOS_SPAN")) span = std::max(2, std::min(8, std::atoi(e)));
  if (lanczos_bytes(n, nl, k, span, b) + 1e9 > avail) return block_lanczos_lean(c, k);
  const int mmax = (int)std::min<int64_t>(n, (int64_t)span * kk + 2 * b);
  const bool dev = dev_svqb && n >= 8 * (int64_t)mmax;
  // row stride padded to whole 128-byte lines so every b-column gather touches whole L2 lines
  const int ld = (mmax + b + 15) / 16 * 16;
  // mixed precision: the FP32-gather products carry rounding noise of about 1e-8 of |theta|, so
  // the Lanczos stops at 1e-7 and the final FP64 sweep corrects the Ritz pairs
  const bool mixed = c->o.precision == 1;
  const double tol = std::max(c->o.eig_tol > 0 ? c->o.eig_tol : 1e-10, mixed ? kMixedTol : 0.0);
  const double eps23 = std::pow(DBL_EPSILON, 2.0 / 3.0);
  const char* prof = std::getenv("VHCI_PROFILE");
  const int plevel = prof ? std::atoi(prof) : 0;
  LWork w;
  VCK(w.Q.reserve((size_t)nl * ld, s));
  VCK(w.HQ.reserve((size_t)nl * ld, s));
  VCK(w.T.reserve((size_t)ld * ld, s));
  VCK(w.Yw.reserve((size_t)ld * ld, s));
  VCK(w.theta.reserve(ld, s));
  VCK(w.Xb.reserve((size_t)rb * kk, s));  // rblk rows: the block each rank gathers at the end
  if (mixed) VCK(w.HXb.reserve((size_t)nl * kk, s));  // the final FP64 sweep's products
  VCK(w.W.reserve((size_t)nl * b, s));
  const int nblk = residual_blocks(nl);
  VCK(w.part.reserve((size_t)nblk * kk, s));
  VCK(w.rn2.reserve(kk, s));
  VCK(w.short_flag.reserve(1, s));
  VCK(cudaMemsetAsync(w.short_flag.p, 0, sizeof(int), s));
  fill_zero(w.Q.p, nl * (int64_t)ld, s);
  VCK(cudaMemsetAsync(w.T.p, 0, (size_t)ld * ld * sizeof(double), s));

  // ---- start block: random combinations of the previous Ritz vectors, else random vectors
  std::vector<double> rnd;
  uint64_t st = 0x9E3779B97F4A7C15ull;
  auto urand = [&]() {
    st = mix64(st + 0x632BE59BD9B4E019ull);
    return ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  auto nrand = [&]() { return std::sqrt(-2.0 * std::log(urand())) * std::cos(6.283185307179586 * urand()); };
  int m = 0, p = 0;
  if (c->nvec > 0 && c->x_rows > 0 && c->x_rows <= n) {
    // start block = X0 R (random R, w0 x b), zero on the new states: the Krylov space it
    // generates contains the previous Ritz vectors after about w0/b steps, and the Krylov-Schur
    // relation holds from the first step on
    const int w0 = std::min(c->nvec, kk);
    rnd.resize((size_t)w0 * b);
    for (auto& x : rnd) x = nrand();
    DBuf<double> R;
    VCK(R.reserve(rnd.size(), s));
    VCK(h2d(c, R.p, rnd.data(), rnd.size() * sizeof(double)));
    // this rank's rows of the previous vectors (held whole): rows r0 .. r0 + xr - 1
    const int64_t xr = std::max<int64_t>(0, std::min<int64_t>(nl, c->x_rows - r0));
    VTRY(gemm_rows(c, c->X.p + (size_t)r0 * c->ldx, c->ldx, R.p, w0, xr, w0, b, 1.0, 0.0, w.W.p, b));
    if (xr < nl) fill_zero(w.W.p + (size_t)xr * b, (nl - xr) * (int64_t)b, s);
    VTRY(svqb_small(c, w, nl, w.W.p, b, b, w.Q.p, ld, &p));
    VCK(cudaStreamSynchronize(s));
    R.release(s);
    if (p == 0) return fail(c, VHCI_E_NOT_CONVERGED, "empty start block");
  } else {
    random_rows(r0, nl, b, rnd);
    VCK(h2d(c, w.W.p, rnd.data(), rnd.size() * sizeof(double)));
    VTRY(svqb_small(c, w, nl, w.W.p, b, b, w.Q.p, ld, &p));
    if (p == 0) return fail(c, VHCI_E_NOT_CONVERGED, "empty start block");
  }

  std::vector<double> th(ld), rn(kk);
  const int maxcyc = c->o.eig_maxit > 0 ? c->o.eig_maxit : 1000;
  auto t_start = std::chrono::steady_clock::now();
  double t_spmm = 0, t_orth = 0, t_rr = 0;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto msince = [&](std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(now() - t0).count();
  };
  int steps = 0;
  for (int cyc = 0; cyc < maxcyc; ++cyc) {
    // ---- expansion
    bool exhausted = (p == 0);
    while (p > 0) {
      auto t0 = now();
      VTRY(apply_h_l(c, w, w.Q.p + m, ld, p, w.HQ.p + m, ld));
      t_spmm += msince(t0);
      t0 = now();
      ++steps;
      // T[0:m+p, m:m+p] = Q^T (H Q_new)
      VTRY(gemm_gram(c, w, w.Q.p, ld, w.HQ.p + m, ld, nl, m + p, p, 1.0, 0.0, w.T.p + (size_t)m * ld, ld));
      m += p;
      if (m + b > mmax || m >= n) {
        if (plevel) { cudaStreamSynchronize(s); t_orth += msince(t0); }
        break;
      }
      // next block: W = H Q_new - Q T[:, new]; second Gram-Schmidt pass; SVQB
      copy_cols(w.HQ.p + (m - p), ld, w.W.p, b, nl, p, s);
      VCK(w.S.reserve((size_t)std::max(m, b) * p, s));
      VTRY(gemm_rows_gram(c, w, w.Q.p, ld, w.T.p + (size_t)(m - p) * ld, ld, nl, m, p, w.W.p, b,
                          w.S.p, m));
      VTRY(gemm_rows(c, w.Q.p, ld, w.S.p, m, nl, m, p, -1.0, 1.0, w.W.p, b));
      int p2 = p;
      if (dev) VTRY(svqb_dev(c, w, nl, w.W.p, b, p, w.Q.p + m, ld));
      else VTRY(svqb_small(c, w, nl, w.W.p, b, p, w.Q.p + m, ld, &p2));
      t_orth += msince(t0);
      p = p2;
      if (p == 0) { exhausted = true; break; }
    }
    // ---- Rayleigh-Ritz on T[0:m, 0:m]
    auto t0 = now();
    c->stats.eig_iterations += 1;
    VCK(cudaMemcpy2DAsync(w.Yw.p, ld * sizeof(double), w.T.p, ld * sizeof(double),
                          m * sizeof(double), m, cudaMemcpyDeviceToDevice, s));
    VTRY(syevd_l(c, w.Yw.p, m, ld, w.theta.p));
    if (dev) {  // a block that lost rank on the device: redo with the host factorisation
      int short_rank = 0;
      VCK(d2h(c, &short_rank, w.short_flag.p, sizeof(int)));
      VCK(cudaStreamSynchronize(s));
      if (short_rank) {
        w.release(s);
        return block_lanczos_impl(c, k, false);
      }
    }
    // one projected solution for every rank: rank 0's
    VTRY(comm_bcast0(c, w.Yw.p, (int64_t)ld * m));
    VTRY(comm_bcast0(c, w.theta.p, m));
    const int nk = std::min(kk, m);
    VTRY(gemm_rows(c, w.Q.p, ld, w.Yw.p, ld, nl, m, nk, 1.0, 0.0, w.Xb.p, kk));
    // Residuals from the Krylov relation H Q = Q T + W E_last^T, where W = (I - Q Q^T) H Q_last is
    // the pending block (formed here; the restart continues from it): the residual of Ritz pair
    // (theta_j, y_j) is W y_j[last block rows], so ||r_j||^2 = y_last^T (W^T W) y_last.  With the
    // full (two-pass) orthogonalisation the relation holds to rounding, far below the tolerance.
    // The whole space (m = n) or an invariant subspace (exhausted) leaves no residual.
    // Mixed precision keeps the explicit residuals ||H x - theta x|| from the rotated products:
    // its FP32-gather products carry rounding noise of about 1e-8 relative, and the Krylov relation
    // (exact for the products as computed within one cycle) does not carry that noise across the
    // restarts' coupling terms, so it can stall at the 1e-7 tolerance.
    const int pw = (!exhausted && m < n && !mixed) ? p : 0;
    std::fill(rn.begin(), rn.end(), 0.0);
    VCK(d2h(c, th.data(), w.theta.p, nk * sizeof(double)));
    if (mixed) {
      VTRY(gemm_rows(c, w.HQ.p, ld, w.Yw.p, ld, nl, m, nk, 1.0, 0.0, w.HXb.p, kk));
      residual_norms(w.Xb.p, w.HXb.p, nl, kk, nk, w.theta.p, w.part.p, nblk, w.rn2.p, s);
      VTRY(comm_sum(c, w.rn2.p, nk));
      VCK(d2h(c, rn.data(), w.rn2.p, nk * sizeof(double)));
      VCK(cudaStreamSynchronize(s));
    } else if (pw > 0) {
      copy_cols(w.HQ.p + (m - pw), ld, w.W.p, b, nl, pw, s);
      VCK(w.S.reserve((size_t)std::max(m, b) * pw, s));
      VTRY(gemm_rows_gram(c, w, w.Q.p, ld, w.T.p + (size_t)(m - pw) * ld, ld, nl, m, pw, w.W.p, b,
                          w.S.p, m));
      VTRY(gemm_rows(c, w.Q.p, ld, w.S.p, m, nl, m, pw, -1.0, 1.0, w.W.p, b));
      VCK(w.M.reserve((size_t)pw * pw, s));
      VTRY(gemm_gram(c, w, w.W.p, b, w.W.p, b, nl, pw, pw, 1.0, 0.0, w.M.p, pw));
      std::vector<double> G((size_t)pw * pw), Yl((size_t)pw * nk);
      VCK(d2h(c, G.data(), w.M.p, G.size() * sizeof(double)));
      VCK(cudaMemcpy2DAsync(Yl.data(), pw * sizeof(double), w.Yw.p + (m - pw), ld * sizeof(double),
                            pw * sizeof(double), nk, cudaMemcpyDeviceToHost, s));
      VCK(cudaStreamSynchronize(s));
      for (int j = 0; j < nk; ++j) {
        const double* y = Yl.data() + (size_t)j * pw;
        double q = 0.0;
        for (int a = 0; a < pw; ++a) {
          double ga = 0.0;
          for (int e = 0; e < pw; ++e) ga += G[(size_t)e * pw + a] * y[e];
          q += y[a] * ga;
        }
        rn[j] = q;
      }
    } else {
      VCK(cudaStreamSynchronize(s));
    }
    const int keff = std::min(k, nk);
    // Mixed precision measures the residual against the spectrum's scale (the largest |Ritz
    // value| of this cycle) instead of |theta|: the FP32 gathers leave a noise floor proportional
    // to ||H||, which a pair with small |theta| cannot get under; the FP64 sweep refines the pairs.
    double scale = 0.0;
    if (mixed) {
      double tl = 0.0;
      VCK(d2h(c, &tl, w.theta.p + (m - 1), sizeof(double)));
      scale = std::max(std::fabs(th[0]), std::fabs(tl));
    }
    auto thresh = [&](int j) { return tol * std::max({eps23, std::fabs(th[j]), scale}); };
    int nconv = 0;
    double rmax = 0.0;
    for (int j = 0; j < keff; ++j) {
      const double r = std::sqrt(std::max(rn[j], 0.0));
      rmax = std::max(rmax, r);
      if (r <= thresh(j)) ++nconv;
    }
    t_rr += msince(t0);
    if (plevel >= 2)
      std::fprintf(stderr, "  lanczos cycle %d m %d b %d converged %d/%d max|r| %.3e\n", cyc, m, b,
                   nconv, keff, rmax);
    if (plevel >= 3)
      for (int j = 0; j < keff; ++j)
        if (!(std::sqrt(std::max(rn[j], 0.0)) <= thresh(j)))
          std::fprintf(stderr, "    pair %d theta %.10e |r|^2 %.3e\n", j, th[j], rn[j]);
    if (nconv == keff || m >= n || exhausted) {
      if (nconv < keff && !(m >= n || exhausted))
        return fail(c, VHCI_E_NOT_CONVERGED, "Error: Eigenvalues did not converge.");
      if (plevel)
        std::fprintf(stderr, "lanczos n %lld k %d b %d cycles %d steps %d ms: spmm %.1f orth %.1f rr %.1f total %.1f\n",
                     (long long)n, k, b, cyc + 1, steps, t_spmm, t_orth, t_rr, msince(t_start));
      if (mixed) VTRY(fp64_sweep(c, w, kk, nk, std::min(k, nk), ld, th));
      VTRY(publish_ritz(c, w.Xb, kk, nk, th));  // the old X buffer is released with w
      w.release(s);
      return VHCI_OK;
    }
    // ---- thick restart: keep the Ritz block, continue from the pending block W (formed above
    // with the residuals, or here in mixed precision, whose rotated products are kept with it)
    t0 = now();
    if (mixed) {
      copy_cols(w.HQ.p + (m - p), ld, w.W.p, b, nl, p, s);
      VCK(w.S.reserve((size_t)std::max(m, b) * p, s));
      VTRY(gemm_rows_gram(c, w, w.Q.p, ld, w.T.p + (size_t)(m - p) * ld, ld, nl, m, p, w.W.p, b,
                          w.S.p, m));
      VTRY(gemm_rows(c, w.Q.p, ld, w.S.p, m, nl, m, p, -1.0, 1.0, w.W.p, b));
      copy_cols(w.HXb.p, kk, w.HQ.p, ld, nl, nk, s);
    }
    copy_cols(w.Xb.p, kk, w.Q.p, ld, nl, nk, s);
    int p2 = p;
    if (dev) VTRY(svqb_dev(c, w, nl, w.W.p, b, p, w.Q.p + nk, ld));
    else VTRY(svqb_small(c, w, nl, w.W.p, b, p, w.Q.p + nk, ld, &p2));
    std::vector<double> Th((size_t)ld * nk, 0.0);
    for (int j = 0; j < nk; ++j) Th[(size_t)j * ld + j] = th[j];
    VCK(cudaMemsetAsync(w.T.p, 0, (size_t)ld * ld * sizeof(double), s));
    VCK(h2d(c, w.T.p, Th.data(), Th.size() * sizeof(double)));
    m = nk;
    p = p2;
    t_rr += msince(t0);
    if (p == 0) {  // the kept block is invariant: one more Rayleigh-Ritz finishes
      exhausted = true;
    }
    if (exhausted) {
      if (mixed) VTRY(fp64_sweep(c, w, kk, nk, std::min(k, nk), ld, th));
      VTRY(publish_ritz(c, w.Xb, kk, nk, th));  // the old X buffer is released with w
      w.release(s);
      return VHCI_OK;
    }
  }
  w.release(s);
  return fail(c, VHCI_E_NOT_CONVERGED, "Error: Eigenvalues did not converge.");
}


// Memory-lean block Lanczos for bases whose Hamiltonian leaves too little device memory for the
// stored H Q blocks and Ritz blocks: the same thick-restart method (subspace 2 kk + 2 b), but
//   * only Q is stored; each step's product H Q_new lives in one n x b buffer, from which the new
//     column of T = Q^T H Q and the next block are formed at once;
//   * convergence is judged from the Krylov relation H Q = Q T + W E_last^T (W: the pending block,
//     orthogonal to Q): the residual of Ritz pair (theta_j, y_j) is W (y_j restricted to the last
//     block), so ||r_j||^2 = y_last^T (W^T W) y_last needs only a p x p Gram matrix;
//   * Ritz vectors are formed in place in Q, in row chunks, and a claimed convergence is confirmed
//     with explicit residuals H x - theta x, block by block, before returning.
int block_lanczos_lean(vhci_ctx* c, int k) {
  const int64_t n = c->n;
  const int64_t nl = c->nrow, r0 = c->row0, rb = std::max(c->rblk, nl);
  cudaStream_t s = c->st;
  const int guard = lanczos_guard(k);
  const int kk = (int)std::min<int64_t>(n, k + guard);
  const int b = lanczos_block(n);
  const int span = 2;
  const int mmax = (int)std::min<int64_t>(n, (int64_t)span * kk + 2 * b);
  const int ld = (mmax + b + 15) / 16 * 16;
  const double tol = c->o.eig_tol > 0 ? c->o.eig_tol : 1e-10;
  const double eps23 = std::pow(DBL_EPSILON, 2.0 / 3.0);
  const char* prof = std::getenv("VHCI_PROFILE");
  const int plevel = prof ? std::atoi(prof) : 0;
  const int64_t chunk = std::max<int64_t>(1024, (int64_t)(2.5e8 / (8.0 * kk)));
  LWork w;  // Q, T, Yw, theta, W (pending block), HQ (rows x b product), Xb (rotation chunk)
  w.exact = true;  // no final sweep here: FP64 gathers throughout, also in mixed precision
  VCK(w.Q.reserve((size_t)nl * ld, s));
  VCK(w.HQ.reserve((size_t)nl * b, s));
  VCK(w.W.reserve((size_t)nl * b, s));
  VCK(w.Xb.reserve((size_t)std::max<int64_t>(1, std::min<int64_t>(nl, chunk)) * kk, s));
  VCK(w.T.reserve((size_t)ld * ld, s));
  VCK(w.Yw.reserve((size_t)ld * ld, s));
  VCK(w.theta.reserve(ld, s));
  const int nblk = residual_blocks(nl);
  VCK(w.part.reserve((size_t)nblk * b, s));
  VCK(w.rn2.reserve(kk, s));
  fill_zero(w.Q.p, nl * (int64_t)ld, s);
  VCK(cudaMemsetAsync(w.T.p, 0, (size_t)ld * ld * sizeof(double), s));

  // start block, as in block_lanczos
  uint64_t st = 0x9E3779B97F4A7C15ull;
  auto urand = [&]() {
    st = mix64(st + 0x632BE59BD9B4E019ull);
    return ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  auto nrand = [&]() { return std::sqrt(-2.0 * std::log(urand())) * std::cos(6.283185307179586 * urand()); };
  int m = 0, p = 0;
  std::vector<double> rnd;
  if (c->nvec > 0 && c->x_rows > 0 && c->x_rows <= n) {
    const int w0 = std::min(c->nvec, kk);
    rnd.resize((size_t)w0 * b);
    for (auto& x : rnd) x = nrand();
    DBuf<double> R;
    VCK(R.reserve(rnd.size(), s));
    VCK(h2d(c, R.p, rnd.data(), rnd.size() * sizeof(double)));
    const int64_t xr = std::max<int64_t>(0, std::min<int64_t>(nl, c->x_rows - r0));
    VTRY(gemm_rows(c, c->X.p + (size_t)r0 * c->ldx, c->ldx, R.p, w0, xr, w0, b, 1.0, 0.0, w.W.p, b));
    if (xr < nl) fill_zero(w.W.p + (size_t)xr * b, (nl - xr) * (int64_t)b, s);
    VTRY(svqb_small(c, w, nl, w.W.p, b, b, w.Q.p, ld, &p));
    VCK(cudaStreamSynchronize(s));
    R.release(s);
  } else {
    random_rows(r0, nl, b, rnd);
    VCK(h2d(c, w.W.p, rnd.data(), rnd.size() * sizeof(double)));
    VTRY(svqb_small(c, w, nl, w.W.p, b, b, w.Q.p, ld, &p));
  }
  if (p == 0) return fail(c, VHCI_E_NOT_CONVERGED, "empty start block");
  // the previous Ritz block is no longer needed: its memory goes to the Krylov basis
  c->X.release(s);
  c->nvec = 0;
  c->x_rows = 0;

  std::vector<double> th(ld), rn(kk), G, Yl;
  // Q[:, 0:nk] = Q[:, 0:m] Y[0:m, 0:nk], in row chunks through w.Xb
  auto rotate = [&](int mm, int nk) -> int {
    for (int64_t q0 = 0; q0 < nl; q0 += chunk) {
      const int64_t rows = std::min(chunk, nl - q0);
      VTRY(gemm_rows(c, w.Q.p + (size_t)q0 * ld, ld, w.Yw.p, ld, rows, mm, nk, 1.0, 0.0, w.Xb.p, nk));
      VCK(cudaMemcpy2DAsync(w.Q.p + (size_t)q0 * ld, ld * sizeof(double), w.Xb.p,
                            nk * sizeof(double), nk * sizeof(double), rows,
                            cudaMemcpyDeviceToDevice, s));
    }
    return VHCI_OK;
  };
  // the Ritz vectors, rotated into Q[:, 0:nk], become the context's vectors
  auto finish = [&](int nk) -> int {
    w.HQ.release(s);
    w.W.release(s);
    w.Xb.release(s);
    DBuf<double> out;
    VCK(out.reserve((size_t)rb * kk, s));
    copy_cols(w.Q.p, ld, out.p, kk, nl, nk, s);
    VTRY(publish_ritz(c, out, kk, nk, th));
    out.release(s);
    w.release(s);
    return VHCI_OK;
  };

  const int maxcyc = c->o.eig_maxit > 0 ? c->o.eig_maxit : 1000;
  auto t_start = std::chrono::steady_clock::now();
  int steps = 0;
  for (int cyc = 0; cyc < maxcyc; ++cyc) {
    bool exhausted = false;
    int plast = 0;  // width of the block whose product formed the pending W
    while (true) {
      VTRY(apply_h_l(c, w, w.Q.p + m, ld, p, w.HQ.p, b));
      ++steps;
      VTRY(gemm_gram(c, w, w.Q.p, ld, w.HQ.p, b, nl, m + p, p, 1.0, 0.0, w.T.p + (size_t)m * ld, ld));
      m += p;
      plast = p;
      // pending block W = H Q_new - Q T[:, new], second Gram-Schmidt pass
      VCK(cudaMemcpyAsync(w.W.p, w.HQ.p, (size_t)nl * b * sizeof(double), cudaMemcpyDeviceToDevice, s));
      VCK(w.S.reserve((size_t)m * p, s));
      VTRY(gemm_rows_gram(c, w, w.Q.p, ld, w.T.p + (size_t)(m - p) * ld, ld, nl, m, p, w.W.p, b,
                          w.S.p, m));
      VTRY(gemm_rows(c, w.Q.p, ld, w.S.p, m, nl, m, p, -1.0, 1.0, w.W.p, b));
      if (m + b > mmax || m >= n) break;
      int p2 = 0;
      VTRY(svqb_small(c, w, nl, w.W.p, b, p, w.Q.p + m, ld, &p2));
      if (p2 == 0) { exhausted = true; break; }
      p = p2;
    }
    // Rayleigh-Ritz
    c->stats.eig_iterations += 1;
    VCK(cudaMemcpy2DAsync(w.Yw.p, ld * sizeof(double), w.T.p, ld * sizeof(double),
                          m * sizeof(double), m, cudaMemcpyDeviceToDevice, s));
    VTRY(syevd_l(c, w.Yw.p, m, ld, w.theta.p));
    VTRY(comm_bcast0(c, w.Yw.p, (int64_t)ld * m));
    VTRY(comm_bcast0(c, w.theta.p, m));
    const int nk = std::min(kk, m);
    const int keff = std::min(k, nk);
    VCK(d2h(c, th.data(), w.theta.p, m * sizeof(double)));
    // residual estimates from the pending block: G = W^T W (plast x plast), Y's last-block rows
    VCK(w.S.reserve((size_t)plast * plast, s));
    VTRY(gemm_gram(c, w, w.W.p, b, w.W.p, b, nl, plast, plast, 1.0, 0.0, w.S.p, plast));
    G.resize((size_t)plast * plast);
    Yl.resize((size_t)plast * nk);
    VCK(d2h(c, G.data(), w.S.p, G.size() * sizeof(double)));
    VCK(cudaMemcpy2DAsync(Yl.data(), plast * sizeof(double), w.Yw.p + (m - plast), ld * sizeof(double),
                          plast * sizeof(double), nk, cudaMemcpyDeviceToHost, s));
    VCK(cudaStreamSynchronize(s));
    int nconv = 0;
    double rmax = 0.0;
    for (int j = 0; j < keff; ++j) {
      const double* y = Yl.data() + (size_t)j * plast;
      double r2 = 0.0;
      for (int a = 0; a < plast; ++a)
        for (int q = 0; q < plast; ++q) r2 += y[a] * G[(size_t)q * plast + a] * y[q];
      const double r = std::sqrt(std::max(r2, 0.0));
      rmax = std::max(rmax, r);
      if (r <= tol * std::max(eps23, std::fabs(th[j]))) ++nconv;
    }
    if (plevel >= 2)
      std::fprintf(stderr, "  lean lanczos cycle %d m %d converged(est) %d/%d max|r| %.3e\n", cyc, m,
                   nconv, keff, rmax);
    const bool full = m >= n || exhausted;
    VTRY(rotate(m, nk));
    bool done = full;
    if (!full && nconv == keff) {
      // confirm with explicit residuals, b Ritz vectors at a time
      done = true;
      for (int j0 = 0; j0 < keff && done; j0 += b) {
        const int bw = std::min(b, keff - j0);
        // compact copy (w.Xc) and product both n x bw
        VTRY(apply_h_l(c, w, w.Q.p + j0, ld, bw, w.HQ.p, bw));
        residual_norms(w.Xc.p, w.HQ.p, nl, bw, bw, w.theta.p + j0, w.part.p, nblk, w.rn2.p + j0, s);
        VTRY(comm_sum(c, w.rn2.p + j0, bw));
        VCK(d2h(c, rn.data() + j0, w.rn2.p + j0, bw * sizeof(double)));
        VCK(cudaStreamSynchronize(s));
        for (int j = j0; j < j0 + bw; ++j)
          if (std::sqrt(std::max(rn[j], 0.0)) > tol * std::max(eps23, std::fabs(th[j]))) done = false;
      }
    }
    if (done) {
      if (plevel)
        std::fprintf(stderr, "lanczos(lean) n %lld k %d b %d span %d cycles %d steps %d ms total %.1f\n",
                     (long long)n, k, b, span, cyc + 1, steps,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
      return finish(nk);
    }
    // thick restart: kept Ritz vectors Q[:, 0:nk] (already rotated), then the pending block
    int p2 = 0;
    VTRY(svqb_small(c, w, nl, w.W.p, b, plast, w.Q.p + nk, ld, &p2));
    std::vector<double> Th((size_t)ld * nk, 0.0);
    for (int j = 0; j < nk; ++j) Th[(size_t)j * ld + j] = th[j];
    VCK(cudaMemsetAsync(w.T.p, 0, (size_t)ld * ld * sizeof(double), s));
    VCK(h2d(c, w.T.p, Th.data(), Th.size() * sizeof(double)));
    m = nk;
    p = p2;
    if (p == 0) return finish(nk);  // invariant: the rotated block is exact
  }
  w.release(s);
  return fail(c, VHCI_E_NOT_CONVERGED, "Error: Eigenvalues did not converge.");
}

}  // namespace vhci
