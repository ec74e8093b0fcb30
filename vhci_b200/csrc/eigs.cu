// Lowest eigenpairs of the sparse Hamiltonian (reference: SparseDiagonalize / DenseDiagonalize,
// Ham.cpp:347-379).  Small bases (and the first heat-bath step over the initial basis) use a dense
// symmetric eigensolve on the device (cuSOLVER syevd over the matrix expanded from its CSR form);
// larger ones use the block thick-restart Lanczos of lanczos.cu, whose projections run on the
// FP64 tensor pipe (k_proj.cu).  Convergence follows the reference eigensolver's rule
// ||r_j|| <= tol * max(eps^(2/3), |theta_j|) for the wanted pairs (tol = 1e-10, Ham.cpp:363).
#include <algorithm>
#include <cstdlib>
#include <string>
#include <vector>

#include "internal.h"

namespace vhci {

namespace {

// X (n x keep, row-major) = the first `keep` columns of the column-major n x n matrix A.
__global__ void k_cols_to_rows(const double* __restrict__ A, int64_t n, int keep,
                               double* __restrict__ X) {
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n * keep;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / keep;
    const int j = (int)(idx - i * keep);
    X[idx] = A[i + (int64_t)j * n];
  }
}

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

}  // namespace

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

int dense_eigs(vhci_ctx* c, int keep) {
  const int64_t n = c->n;
  if (!c->h_valid || c->h_rows) VTRY(build_h(c, true));  // the dense solve needs every row
  keep = (int)std::min<int64_t>(keep, n);
  DBuf<double> A, w;
  VCK(A.reserve((size_t)n * n, c->st));
  VCK(w.reserve(n, c->st));
  dense_from_csr(n, c->rowptr.p, c->col.p, c->o.precision == 1 ? nullptr : c->val.p,
                 c->o.precision == 1 ? c->valf.p : nullptr, c->diag.p, A.p, c->st);
  VTRY(syevd(c, A.p, (int)n, (int)n, w.p));
  VCK(c->X.reserve((size_t)n * keep, c->st));
  {
    const int64_t tot = n * keep;
    const int g = (int)std::min<int64_t>(148 * 16, std::max<int64_t>(1, (tot + 255) / 256));
    note_launch();
    k_cols_to_rows<<<g, 256, 0, c->st>>>(A.p, n, keep, c->X.p);
  }
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
  const int r = dense_path(n, k) ? dense_eigs(c, kk) : block_lanczos(c, k);
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
  if (is_sharded(c)) return fail(c, VHCI_E_STATE, "vhci_apply_h on a sharded context");
  if (!c->h_valid || c->h_rows) VTRY(build_h(c, true));
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
