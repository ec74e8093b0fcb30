// Lowest eigenpairs of the sparse Hamiltonian (reference: SparseDiagonalize / DenseDiagonalize,
// Ham.cpp:347-379).  Small bases use a dense symmetric eigensolve on the device.  Larger ones use
// block Davidson with a diagonal preconditioner:
//   * SpMM (k_ham.cu) applies H to a block of vectors stored row-major (N x ld), so every
//     matrix entry gathers one contiguous vector row;
//   * Gram matrices, Rayleigh-Ritz projections and Ritz-vector updates are FP64 GEMMs (cuBLAS);
//   * the projected problem and the block orthonormalisation (SVQB) use cuSOLVER syevd;
//   * convergence uses the reference eigensolver's rule ||r_j|| <= tol * max(eps^(2/3), |theta_j|)
//     for the wanted pairs (tol = 1e-10 by default, Ham.cpp:363).
// HCI iterations warm-start from the previous Ritz vectors, zero-extended over the new states.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace vhci {

namespace {

// Optional section timing of the eigensolver (environment variable VHCI_PROFILE=1|2); it
// synchronises the stream at section boundaries, so it is off by default.
struct Prof {
  int level = 0;
  double t[8] = {0};
  std::chrono::steady_clock::time_point last;
  cudaStream_t s = nullptr;
  explicit Prof(cudaStream_t st) : s(st) {
    const char* e = std::getenv("VHCI_PROFILE");
    level = e ? std::atoi(e) : 0;
    last = std::chrono::steady_clock::now();
  }
  void tick(int sec) {
    if (!level) return;
    cudaStreamSynchronize(s);
    auto now = std::chrono::steady_clock::now();
    t[sec] += std::chrono::duration<double, std::milli>(now - last).count();
    last = now;
  }
};

struct Work {
  DBuf<double> V, HV, Xn, HXn, Tb, Tb2, G, Yw, theta, S, part, rn2, M;
  DBuf<int> cols;
  void release(cudaStream_t s) {
    V.release(s); HV.release(s); Xn.release(s); HXn.release(s); Tb.release(s); Tb2.release(s);
    G.release(s); Yw.release(s); theta.release(s); S.release(s); part.release(s); rn2.release(s);
    M.release(s); cols.release(s);
  }
};

int syevd(vhci_ctx* c, double* A, int m, int lda, double* w) {
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
  if (info != 0) return fail(c, VHCI_E_NOT_CONVERGED, "dense eigensolver failed, info=" + std::to_string(info));
  return VHCI_OK;
}

// Orthonormalise nb columns of a row-major block (B, ld) into (out, ldo) by SVQB; columns whose
// scaled Gram eigenvalue falls below 1e-12 of the largest are dropped.  Returns the rank in *r.
int svqb(vhci_ctx* c, Work& w, int64_t n, const double* B, int ld, int nb, double* out, int ldo,
         int* r) {
  *r = 0;
  if (nb <= 0) return VHCI_OK;
  const double one = 1.0, zero = 0.0;
  VCK(w.S.reserve((size_t)nb * nb, c->st));
  VBL(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, nb, nb, (int)n, &one, B, ld, B, ld, &zero,
                  w.S.p, nb));
  std::vector<double> S((size_t)nb * nb);
  VCK(d2h(c, S.data(), w.S.p, S.size() * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  std::vector<double> d(nb);
  for (int i = 0; i < nb; ++i) {
    const double s = S[(size_t)i * nb + i];
    d[i] = s > 1e-300 ? 1.0 / std::sqrt(s) : 0.0;
  }
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) S[(size_t)j * nb + i] *= d[i] * d[j];
  VCK(h2d(c, w.S.p, S.data(), S.size() * sizeof(double)));
  DBuf<double> lam;
  VCK(lam.reserve(nb, c->st));
  VTRY(syevd(c, w.S.p, nb, nb, lam.p));
  std::vector<double> U((size_t)nb * nb), L(nb);
  VCK(d2h(c, U.data(), w.S.p, U.size() * sizeof(double)));
  VCK(d2h(c, L.data(), lam.p, nb * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  lam.release(c->st);
  const double lmax = L[nb - 1];
  std::vector<int> keep;
  for (int j = nb - 1; j >= 0; --j)
    if (L[j] > 1e-12 * lmax && L[j] > 0) keep.push_back(j);
  const int rr = (int)keep.size();
  if (rr == 0) return VHCI_OK;
  std::vector<double> Mh((size_t)nb * rr);
  for (int q = 0; q < rr; ++q) {
    const int j = keep[q];
    const double s = 1.0 / std::sqrt(L[j]);
    for (int i = 0; i < nb; ++i) Mh[(size_t)q * nb + i] = d[i] * U[(size_t)j * nb + i] * s;
  }
  VCK(w.M.reserve(Mh.size(), c->st));
  VCK(h2d(c, w.M.p, Mh.data(), Mh.size() * sizeof(double)));
  // out^T (rr x n) = M^T (rr x nb) * B^T (nb x n)
  VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, rr, (int)n, nb, &one, w.M.p, nb, B, ld, &zero,
                  out, ldo));
  *r = rr;
  return VHCI_OK;
}

// B (nb cols, ld) -= V[:, 0:m] (V^T B), `passes` times (classical Gram-Schmidt; the Davidson
// step interleaves single passes with SVQB, which together re-orthogonalise).
int project_out(vhci_ctx* c, Work& w, int64_t n, const double* V, int ldv, int m, double* B,
                int ld, int nb, int passes = 2) {
  if (m <= 0 || nb <= 0) return VHCI_OK;
  const double one = 1.0, zero = 0.0, mone = -1.0;
  VCK(w.S.reserve((size_t)m * nb, c->st));
  for (int pass = 0; pass < passes; ++pass) {
    VBL(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, m, nb, (int)n, &one, V, ldv, B, ld, &zero,
                    w.S.p, m));
    VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, nb, (int)n, m, &mone, w.S.p, m, V, ldv,
                    &one, B, ld));
  }
  return VHCI_OK;
}

int apply_h(vhci_ctx* c, const double* X, int ldx, int b, double* Y, int ldy) {
  EventPair ev_e0e1;
  VCK(ev_e0e1.create());
  cudaEvent_t e0 = ev_e0e1.a, e1 = ev_e0e1.b;
  VCK(cudaEventRecord(e0, c->st));
  spmm_h(c, X, ldx, b, Y, ldy);
  VCK(cudaEventRecord(e1, c->st));
  VCK(cudaEventSynchronize(e1));
  VCK(cudaGetLastError());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  c->stats.ms_spmm += ms;
  c->stats.spmm_calls += 1;
  c->stats.spmm_cols += b;
  const int64_t sval = c->o.precision == 1 ? 4 : 8;
  c->stats.spmm_gather_bytes += c->nnz * (int64_t)b * 8;
  c->stats.spmm_bytes += c->nnz * (sval + 4) + (c->n + 1) * 8 + c->n * 8 +
                         2 * c->n * (int64_t)b * 8;
  return VHCI_OK;
}

// Orthonormalise p coefficient columns A (m x p, column-major, lda) into Z (m x r, ldz) by SVQB.
int svqb_cols(vhci_ctx* c, Work& w, const double* A, int m, int p, int lda, double* Z, int ldz,
              int* r) {
  *r = 0;
  if (p <= 0 || m <= 0) return VHCI_OK;
  const double one = 1.0, zero = 0.0;
  VCK(w.S.reserve((size_t)p * p, c->st));
  VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, p, p, m, &one, A, lda, A, lda, &zero, w.S.p, p));
  std::vector<double> S((size_t)p * p);
  VCK(d2h(c, S.data(), w.S.p, S.size() * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  std::vector<double> d(p);
  double dmax = 0;
  for (int i = 0; i < p; ++i) dmax = std::max(dmax, S[(size_t)i * p + i]);
  for (int i = 0; i < p; ++i) {
    const double s = S[(size_t)i * p + i];
    d[i] = s > 1e-20 * dmax && s > 1e-300 ? 1.0 / std::sqrt(s) : 0.0;
  }
  for (int j = 0; j < p; ++j)
    for (int i = 0; i < p; ++i) S[(size_t)j * p + i] *= d[i] * d[j];
  VCK(h2d(c, w.S.p, S.data(), S.size() * sizeof(double)));
  DBuf<double> lam;
  VCK(lam.reserve(p, c->st));
  VTRY(syevd(c, w.S.p, p, p, lam.p));
  std::vector<double> U((size_t)p * p), L(p);
  VCK(d2h(c, U.data(), w.S.p, U.size() * sizeof(double)));
  VCK(d2h(c, L.data(), lam.p, p * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  lam.release(c->st);
  const double lmax = L[p - 1];
  std::vector<int> keep;
  for (int j = p - 1; j >= 0; --j)
    if (L[j] > 1e-10 * lmax && L[j] > 0) keep.push_back(j);
  const int rr = (int)keep.size();
  if (rr == 0) return VHCI_OK;
  std::vector<double> Mh((size_t)p * rr);
  for (int q = 0; q < rr; ++q) {
    const int j = keep[q];
    const double s = 1.0 / std::sqrt(L[j]);
    for (int i = 0; i < p; ++i) Mh[(size_t)q * p + i] = d[i] * U[(size_t)j * p + i] * s;
  }
  VCK(w.M.reserve(Mh.size(), c->st));
  VCK(h2d(c, w.M.p, Mh.data(), Mh.size() * sizeof(double)));
  VBL(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, m, rr, p, &one, A, lda, w.M.p, p, &zero, Z, ldz));
  *r = rr;
  return VHCI_OK;
}

// Block Davidson with GD+k restarts: when the subspace is full it is rebuilt from the current
// Ritz block and the previous iteration's Ritz block (orthogonalised against it), which keeps the
// convergence history that a plain thick restart loses.
int davidson(vhci_ctx* c, int k) {
  const int64_t n = c->n;
  const int guard = std::max(4, k / 10);
  const int kk = (int)std::min<int64_t>(n, k + guard);
  const int mmax = (int)std::min<int64_t>(n, 2 * kk + 2 * std::min(k, kk));
  const double one = 1.0, zero = 0.0, mone = -1.0;
  const double tol = c->o.eig_tol > 0 ? c->o.eig_tol : 1e-10;
  const double eps23 = std::pow(DBL_EPSILON, 2.0 / 3.0);
  Work w;
  cudaStream_t s = c->st;
  VCK(w.V.reserve((size_t)n * mmax, s));
  VCK(w.HV.reserve((size_t)n * mmax, s));
  VCK(w.Xn.reserve((size_t)n * kk, s));
  VCK(w.HXn.reserve((size_t)n * kk, s));
  VCK(w.Tb.reserve((size_t)n * kk, s));
  VCK(w.Tb2.reserve((size_t)n * kk, s));
  VCK(w.G.reserve((size_t)mmax * mmax, s));
  VCK(w.Yw.reserve((size_t)mmax * mmax, s));
  VCK(w.theta.reserve(mmax, s));
  DBuf<double> Yp, Z, T1, C1;
  VCK(Yp.reserve((size_t)mmax * kk, s));
  VCK(Z.reserve((size_t)mmax * kk, s));
  VCK(T1.reserve((size_t)mmax * kk, s));
  VCK(C1.reserve((size_t)kk * kk, s));
  const int nblk = residual_blocks(n);
  VCK(w.part.reserve((size_t)nblk * kk, s));
  VCK(w.rn2.reserve(kk, s));
  VCK(w.cols.reserve(kk, s));
  fill_zero(w.V.p, n * (int64_t)mmax, s);

  // ---- initial block: previous Ritz vectors (zero-extended) + unit vectors on low diagonals
  int w0 = 0;
  if (c->nvec > 0 && c->x_rows > 0 && c->x_rows <= n) {
    w0 = std::min(c->nvec, kk);
    copy_cols(c->X.p, c->ldx, w.V.p, mmax, c->x_rows, w0, s);
  }
  const int extra = kk - w0;
  if (extra > 0) {
    std::vector<double> dg(n);
    VCK(d2h(c, dg.data(), c->diag.p, n * sizeof(double)));
    VCK(cudaStreamSynchronize(s));
    const int64_t from = (w0 > 0) ? c->x_rows : 0;
    std::vector<int64_t> idx;
    for (int64_t i = from; i < n; ++i) idx.push_back(i);
    if ((int64_t)idx.size() < extra)
      for (int64_t i = 0; i < from; ++i) idx.push_back(i);
    const int take = (int)std::min<int64_t>(extra, (int64_t)idx.size());
    std::partial_sort(idx.begin(), idx.begin() + take, idx.end(), [&](int64_t a, int64_t b) {
      return dg[a] < dg[b] || (dg[a] == dg[b] && a < b);
    });
    DBuf<int64_t> rows;
    VCK(rows.reserve(take, s));
    VCK(h2d(c, rows.p, idx.data(), take * sizeof(int64_t)));
    set_unit_rows(w.V.p, mmax, w0, rows.p, take, s);
    VCK(cudaStreamSynchronize(s));
    rows.release(s);
  }
  int m = 0;
  VTRY(svqb(c, w, n, w.V.p, mmax, kk, w.Tb2.p, kk, &m));
  copy_cols(w.Tb2.p, kk, w.V.p, mmax, n, m, s);
  {
    int m2 = 0;
    VTRY(svqb(c, w, n, w.V.p, mmax, m, w.Tb2.p, kk, &m2));
    copy_cols(w.Tb2.p, kk, w.V.p, mmax, n, m2, s);
    m = m2;
  }
  if (m == 0) return fail(c, VHCI_E_NOT_CONVERGED, "empty initial subspace");
  VTRY(apply_h(c, w.V.p, mmax, m, w.HV.p, mmax));
  VBL(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, m, m, (int)n, &one, w.V.p, mmax, w.HV.p, mmax,
                  &zero, w.G.p, mmax));

  std::vector<double> th(mmax), rn(kk);
  Prof pf(s);
  pf.tick(7);
  bool have_prev = false;
  int kp = 0;  // columns of the previous Ritz block held in Yp
  const int maxit = c->o.eig_maxit > 0 ? c->o.eig_maxit : 1000;
  for (int it = 0; it < maxit; ++it) {
    c->stats.eig_iterations += 1;
    VCK(cudaMemcpy2DAsync(w.Yw.p, mmax * sizeof(double), w.G.p, mmax * sizeof(double),
                          m * sizeof(double), m, cudaMemcpyDeviceToDevice, s));
    VTRY(syevd(c, w.Yw.p, m, mmax, w.theta.p));
    pf.tick(0);
    const int nk = std::min(kk, m);
    VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, nk, (int)n, m, &one, w.Yw.p, mmax, w.V.p,
                    mmax, &zero, w.Xn.p, kk));
    VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, nk, (int)n, m, &one, w.Yw.p, mmax, w.HV.p,
                    mmax, &zero, w.HXn.p, kk));
    residual_norms(w.Xn.p, w.HXn.p, n, kk, nk, w.theta.p, w.part.p, nblk, w.rn2.p, s);
    VCK(d2h(c, th.data(), w.theta.p, nk * sizeof(double)));
    VCK(d2h(c, rn.data(), w.rn2.p, nk * sizeof(double)));
    VCK(cudaStreamSynchronize(s));
    pf.tick(1);
    const int keff = std::min(k, nk);
    std::vector<int> cols;
    for (int j = 0; j < keff; ++j)
      if (!(std::sqrt(std::max(rn[j], 0.0)) <= tol * std::max(eps23, std::fabs(th[j]))))
        cols.push_back(j);
    if (pf.level >= 2) {
      double mx = 0;
      for (int j = 0; j < keff; ++j) mx = std::max(mx, std::sqrt(std::max(rn[j], 0.0)));
      std::fprintf(stderr, "  davidson it %d m %d unconverged %zu max|r| %.3e\n", it, m, cols.size(), mx);
    }
    if (cols.empty() || m >= n) {
      if (pf.level)
        std::fprintf(stderr, "davidson n %lld k %d iters %d ms: rr %.1f ritz %.1f restart %.1f orth %.1f spmm %.1f gram %.1f init %.1f\n",
                     (long long)n, k, it + 1, pf.t[0], pf.t[1], pf.t[2], pf.t[3], pf.t[4], pf.t[5], pf.t[7]);
      VCK(c->X.reserve((size_t)n * kk, s));
      VCK(cudaMemcpyAsync(c->X.p, w.Xn.p, (size_t)n * kk * sizeof(double), cudaMemcpyDeviceToDevice, s));
      c->ldx = kk;
      c->nvec = nk;
      c->x_rows = n;
      c->E.assign(th.begin(), th.begin() + nk);
      VCK(cudaStreamSynchronize(s));
      w.release(s); Yp.release(s); Z.release(s); T1.release(s); C1.release(s);
      return VHCI_OK;
    }
    int nc = (int)cols.size();
    if (m + nc > mmax) {
      // ---- GD+k restart: basis = [current Ritz block, orth(previous Ritz block)]
      int r = 0;
      if (have_prev && kp > 0) {
        for (int pass = 0; pass < 2; ++pass) {
          VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, nk, kp, m, &one, w.Yw.p, mmax, Yp.p,
                          mmax, &zero, C1.p, kk));
          VBL(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, m, kp, nk, &mone, w.Yw.p, mmax, C1.p,
                          kk, &one, Yp.p, mmax));
        }
        VTRY(svqb_cols(c, w, Yp.p, m, kp, mmax, Z.p, mmax, &r));
        r = std::min(r, mmax - nk - 1);
        if (r > 0) {
          VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, r, (int)n, m, &one, Z.p, mmax, w.V.p,
                          mmax, &zero, w.Tb.p, kk));
          VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, r, (int)n, m, &one, Z.p, mmax, w.HV.p,
                          mmax, &zero, w.Tb2.p, kk));
          VBL(cublasDsymm(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, m, r, &one, w.G.p, mmax,
                          Z.p, mmax, &zero, T1.p, mmax));
          VBL(cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, r, r, m, &one, Z.p, mmax, T1.p, mmax,
                          &zero, C1.p, kk));
        }
      }
      copy_cols(w.Xn.p, kk, w.V.p, mmax, n, nk, s);
      copy_cols(w.HXn.p, kk, w.HV.p, mmax, n, nk, s);
      if (r > 0) {
        copy_cols(w.Tb.p, kk, w.V.p + nk, mmax, n, r, s);
        copy_cols(w.Tb2.p, kk, w.HV.p + nk, mmax, n, r, s);
      }
      std::vector<double> Gh((size_t)mmax * (nk + r), 0.0);
      for (int j = 0; j < nk; ++j) Gh[(size_t)j * mmax + j] = th[j];
      if (r > 0) {
        std::vector<double> g22((size_t)kk * r);
        VCK(d2h(c, g22.data(), C1.p, g22.size() * sizeof(double)));
        VCK(cudaStreamSynchronize(s));
        for (int j = 0; j < r; ++j)
          for (int i = 0; i < r; ++i) Gh[(size_t)(nk + j) * mmax + nk + i] = g22[(size_t)j * kk + i];
      }
      VCK(h2d(c, w.G.p, Gh.data(), Gh.size() * sizeof(double)));
      m = nk + r;
      // the current Ritz vectors are now the first nk basis vectors
      std::vector<double> Yh((size_t)mmax * nk, 0.0);
      for (int j = 0; j < nk; ++j) Yh[(size_t)j * mmax + j] = 1.0;
      VCK(h2d(c, Yp.p, Yh.data(), Yh.size() * sizeof(double)));
      kp = nk;
      have_prev = true;
      if (m + nc > mmax) nc = mmax - m;
      if (nc <= 0) return fail(c, VHCI_E_NOT_CONVERGED, "Davidson subspace exhausted");
      pf.tick(2);
    } else {
      // remember this iteration's Ritz coefficients (zero below row m)
      VCK(cudaMemsetAsync(Yp.p, 0, (size_t)mmax * nk * sizeof(double), s));
      VCK(cudaMemcpy2DAsync(Yp.p, mmax * sizeof(double), w.Yw.p, mmax * sizeof(double),
                            m * sizeof(double), nk, cudaMemcpyDeviceToDevice, s));
      kp = nk;
      have_prev = true;
    }
    VCK(h2d(c, w.cols.p, cols.data(), nc * sizeof(int)));
    VCK(w.part.reserve(std::max<size_t>((size_t)nblk * kk, (size_t)correction_scratch(n, nc)), s, false));
    davidson_correction(w.Xn.p, w.HXn.p, kk, c->diag.p, n, w.cols.p, w.theta.p, nc, w.Tb.p, kk,
                        w.part.p, s);
    VTRY(project_out(c, w, n, w.V.p, mmax, m, w.Tb.p, kk, nc, 1));
    int r = 0;
    VTRY(svqb(c, w, n, w.Tb.p, kk, nc, w.Tb2.p, kk, &r));
    VTRY(project_out(c, w, n, w.V.p, mmax, m, w.Tb2.p, kk, r, 1));
    int r2 = 0;
    VTRY(svqb(c, w, n, w.Tb2.p, kk, r, w.V.p + m, mmax, &r2));
    if (r2 == 0) return fail(c, VHCI_E_NOT_CONVERGED, "Davidson stagnated (no new directions)");
    pf.tick(3);
    VTRY(apply_h(c, w.V.p + m, mmax, r2, w.HV.p + m, mmax));
    pf.tick(4);
    VBL(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, m + r2, r2, (int)n, &one, w.V.p, mmax,
                    w.HV.p + m, mmax, &zero, w.G.p + (size_t)m * mmax, mmax));
    pf.tick(5);
    m += r2;
  }
  w.release(s); Yp.release(s); Z.release(s); T1.release(s); C1.release(s);
  return fail(c, VHCI_E_NOT_CONVERGED, "Error: Eigenvalues did not converge.");
}

}  // namespace

int dense_eigs(vhci_ctx* c, int keep) {
  const int64_t n = c->n;
  if (!c->h_valid) VTRY(build_h(c));
  keep = (int)std::min<int64_t>(keep, n);
  DBuf<double> A, w;
  VCK(A.reserve((size_t)n * n, c->st));
  VCK(w.reserve(n, c->st));
  dense_from_csr(n, c->rowptr.p, c->col.p, c->o.precision == 1 ? nullptr : c->val.p,
                 c->o.precision == 1 ? c->valf.p : nullptr, c->diag.p, A.p, c->st);
  VTRY(syevd(c, A.p, (int)n, (int)n, w.p));
  VCK(c->X.reserve((size_t)n * keep, c->st));
  const double one = 1.0, zero = 0.0;
  // X row-major (n x keep) = transpose of the first `keep` eigenvector columns
  VBL(cublasDgeam(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, keep, (int)n, &one, A.p, (int)n, &zero, A.p,
                  keep, c->X.p, keep));
  std::vector<double> wh(keep);
  VCK(d2h(c, wh.data(), w.p, keep * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  A.release(c->st);
  w.release(c->st);
  c->ldx = keep;
  c->nvec = keep;
  c->x_rows = n;
  c->E = wh;
  return VHCI_OK;
}

int eigs(vhci_ctx* c, int k) {
  if (!c->h_valid) VTRY(build_h(c));
  const int64_t n = c->n;
  const int guard = std::max(4, k / 10);
  const int kk = (int)std::min<int64_t>(n, k + guard);
  VCK(cudaEventRecord(c->ev_a, c->st));
  int r;
  const char* which = std::getenv("VHCI_EIGS");
  if (n <= 2000 || n <= 3 * (int64_t)kk + 64) r = dense_eigs(c, kk);
  else if (which && std::string(which) == "davidson") r = davidson(c, k);
  else r = block_lanczos(c, k);
  if (r != VHCI_OK) return r;
  VCK(cudaEventRecord(c->ev_b, c->st));
  VCK(cudaEventSynchronize(c->ev_b));
  c->stats.ms_eigs += event_ms(c);
  return VHCI_OK;
}

}  // namespace vhci

using namespace vhci;

extern "C" vhci_status vhci_apply_h(vhci_ctx* c, const double* X, double* Y, int b) {
  if (!c || !X || !Y || b <= 0) return VHCI_E_INPUT;
  if (!c->h_valid) VTRY(build_h(c));
  const int64_t n = c->n;
  std::vector<double> h((size_t)n * b);
  for (int64_t i = 0; i < n; ++i)
    for (int j = 0; j < b; ++j) h[(size_t)i * b + j] = X[(size_t)j * n + i];
  DBuf<double> dx, dy;
  VCK(dx.reserve(h.size(), c->st));
  VCK(dy.reserve(h.size(), c->st));
  VCK(h2d(c, dx.p, h.data(), h.size() * sizeof(double)));
  VTRY(apply_h(c, dx.p, b, b, dy.p, b));
  VCK(d2h(c, h.data(), dy.p, h.size() * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  dx.release(c->st);
  dy.release(c->st);
  for (int64_t i = 0; i < n; ++i)
    for (int j = 0; j < b; ++j) Y[(size_t)j * n + i] = h[(size_t)i * b + j];
  return VHCI_OK;
}

extern "C" vhci_status vhci_eigs(vhci_ctx* c, int k, double* E) {
  if (!c || k <= 0) return VHCI_E_INPUT;
  VTRY(eigs(c, k));
  if (E)
    for (int j = 0; j < std::min<int>(k, (int)c->E.size()); ++j) E[j] = c->E[j];
  return VHCI_OK;
}
