// Internal entry points shared by the host translation units of the library.
#pragma once

#include <string>

#include "ctx.h"

namespace vhci {

int fail(vhci_ctx* c, int code, const std::string& msg);
int cuda_fail(vhci_ctx* c, cudaError_t e, const char* where);
int blas_fail(vhci_ctx* c, int st, const char* where);

#define VCK(call)                                              \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return ::vhci::cuda_fail(c, e_, #call); \
  } while (0)
#define VBL(call)                                              \
  do {                                                         \
    int s_ = (int)(call);                                      \
    if (s_ != 0) return ::vhci::blas_fail(c, s_, #call);       \
  } while (0)
#define VTRY(call)          \
  do {                      \
    int r_ = (call);        \
    if (r_ != VHCI_OK) return r_; \
  } while (0)

HashView basis_view(vhci_ctx* c);
ConnDev conn_view(vhci_ctx* c);
HBTable hb_view(vhci_ctx* c);

// Reads (and clears) the kernel flag word; returns VHCI_OK or a CUDA error.
int read_flags(vhci_ctx* c, int* flags);
int upload_tables(vhci_ctx* c);
int promote_layout(vhci_ctx* c);
int ensure_hash(vhci_ctx* c, int64_t n_total);
int append_keys(vhci_ctx* c, const uint64_t* dkeys, int64_t m);

// Heat-bath candidate set at threshold eps over the held vectors: sorted keys in c->sel,
// count in c->nsel.  Promotes the key layout and retries when a state needs 8-bit fields.
int generate_new_set(vhci_ctx* c, double eps);

// Builds the Hamiltonian: all rows, or this rank's row block when the context is sharded and the
// eigensolve will be the sparse one (all_rows forces every row, as the dense solve needs).
int build_h(vhci_ctx* c, bool all_rows = false);
// The eigensolve of k pairs over n states is dense (small bases): every rank solves it whole.
bool dense_path(int64_t n, int k);

// ---- collectives of a sharded solve (no-ops on an unsharded context) ----
inline bool is_sharded(const vhci_ctx* c) { return c->comm.nranks > 1; }
// buf (device, count doubles) = its sum over the ranks
int comm_sum(vhci_ctx* c, double* buf, int64_t count);
// recv (device) = the ranks' `bytes`-byte send buffers in rank order
int comm_gather(vhci_ctx* c, const void* send, void* recv, int64_t bytes);
// buf = rank 0's values on every rank
int comm_bcast0(vhci_ctx* c, double* buf, int64_t count);
// Two CUDA events that are destroyed with their scope, so early error returns release them.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t create() {
    cudaError_t e = cudaEventCreate(&a);
    return e == cudaSuccess ? cudaEventCreate(&b) : e;
  }
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Entries of the reference's stored pattern (diagonal + gated pairs, structural zeros included).
bool structural_available(vhci_ctx* c);
int structural_count(vhci_ctx* c, int64_t* out);
// Y = H X on the context's stream, through the column panels when they are built.
void spmm_h(vhci_ctx* c, const double* X, int ldx, int b, double* Y, int ldy);
// Device memory a new allocation can use: free memory plus the pool's idle reserve.
double device_available(vhci_ctx* c);
// Device bytes the block Lanczos needs for k eigenpairs on the current basis with its smallest
// subspace (span 2).
double lanczos_min_bytes(vhci_ctx* c, int k);
// Lowest k eigenpairs; dense_all keeps every eigenpair of a dense solve (first HCI step).
int eigs(vhci_ctx* c, int k);
int dense_eigs(vhci_ctx* c, int keep);
// Block thick-restart Lanczos (lanczos.cu).
int block_lanczos(vhci_ctx* c, int k);
int lanczos_block(int64_t n);
int pt2(vhci_ctx* c, double eps2, double* dE, int64_t* n_pert);

float event_ms(vhci_ctx* c);

// Host<->device copies on the context stream, counted in the statistics.
inline cudaError_t h2d(vhci_ctx* c, void* dst, const void* src, size_t bytes) {
  c->stats.h2d_bytes += (int64_t)bytes;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st);
}
inline cudaError_t d2h(vhci_ctx* c, void* dst, const void* src, size_t bytes) {
  c->stats.d2h_bytes += (int64_t)bytes;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->st);
}

}  // namespace vhci
