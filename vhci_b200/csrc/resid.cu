// Residual norms of caller-supplied eigenpairs with the context's Hamiltonian:
// rnorm[j] = || H x_j - theta_j x_j ||, the quantity the reference's eigensolver tests against its
// tolerance (Ham.cpp:363).  One fused pass: row groups form (H x)_i for a panel of up to 32 columns
// (the SpMM of k_ham.cu), subtract theta x_i, square, and add into per-block partial sums kept in
// scratch memory; a second kernel sums the partials in a fixed order.
#include <algorithm>
#include <mutex>
#include <vector>

#include "internal.h"

namespace vhci {

namespace {

constexpr int kResidThreads = 256;
constexpr int kResidBlocks = 148 * 2;  // partial-sum rows (one per block)

template <int BP, typename VT>
__global__ void __launch_bounds__(kResidThreads) k_resid_fused(
    int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
    const VT* __restrict__ val, const double* __restrict__ diag, const double* __restrict__ X,
    int ldx, int bp, const double* __restrict__ theta, double* __restrict__ part, int ldp) {
  constexpr int G = 32 / BP;
  __shared__ double red[kResidThreads / BP][BP];
  const int lane = threadIdx.x & 31;
  const int grp = lane / BP, cc = lane % BP;
  const bool active = cc < bp;
  const double th = active ? theta[cc] : 0.0;
  double s = 0.0;
  const int64_t stride = (int64_t)gridDim.x * (blockDim.x >> 5) * G;
  for (int64_t i = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * G + grp;
       i < n; i += stride) {
    if (!active) continue;
    const int64_t beg = __ldg(rowptr + i), end = __ldg(rowptr + i + 1);
    double acc = 0.0;
#pragma unroll 4
    for (int64_t e = beg; e < end; ++e) {
      const int j = __ldg(col + e);
      const double v = (double)__ldg(val + e);
      acc = fma(v, __ldg(X + (int64_t)j * ldx + cc), acc);
    }
    const double xi = X[i * ldx + cc];
    const double r = fma(diag[i], xi, acc) - th * xi;
    s = fma(r, r, s);
  }
  // block reduction per column, in a fixed order
  red[threadIdx.x / BP][cc] = active ? s : 0.0;
  __syncthreads();
  if (threadIdx.x < BP) {
    double t = 0.0;
    for (int q = 0; q < kResidThreads / BP; ++q) t += red[q][threadIdx.x];
    if (threadIdx.x < bp) part[(int64_t)blockIdx.x * ldp + threadIdx.x] = t;
  }
}

__global__ void k_resid_finish(const double* __restrict__ part, int nblk, int ldp, int k,
                               double* __restrict__ rnorm) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < k; c += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int q = 0; q < nblk; ++q) t += part[(int64_t)q * ldp + c];
    rnorm[c] = sqrt(t);
  }
}

template <typename VT>
void resid_launch(int64_t n, const int64_t* rowptr, const int32_t* col, const VT* val,
                  const double* diag, const double* X, int ldx, int k, const double* theta,
                  double* part, double* rnorm, cudaStream_t s) {
  for (int c0 = 0; c0 < k; c0 += 32) {
    const int bp = std::min(32, k - c0);
    const int BP = bp <= 8 ? 8 : (bp <= 16 ? 16 : 32);
    double* pp = part + c0;
    if (BP == 8) { note_launch(); k_resid_fused<8, VT><<<kResidBlocks, kResidThreads, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bp, theta + c0, pp, k); }
    else if (BP == 16) { note_launch(); k_resid_fused<16, VT><<<kResidBlocks, kResidThreads, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bp, theta + c0, pp, k); }
    else { note_launch(); k_resid_fused<32, VT><<<kResidBlocks, kResidThreads, 0, s>>>(n, rowptr, col, val, diag, X + c0, ldx, bp, theta + c0, pp, k); }
  }
  note_launch();
  k_resid_finish<<<(k + 127) / 128, 128, 0, s>>>(part, kResidBlocks, k, k, rnorm);
}

}  // namespace

// Residual norms for k device-resident vectors X (n x k row-major, ld = k) with device theta;
// `part` is scratch of resid_scratch_elems(k) doubles.
int64_t resid_scratch_elems(int k) { return (int64_t)kResidBlocks * k; }

void residual_norms_fused(vhci_ctx* c, const double* X, int k, const double* theta, double* part,
                          double* rnorm) {
  if (c->o.precision == 1)
    resid_launch<float>(c->n, c->rowptr.p, c->col.p, c->valf.p, c->diag.p, X, k, k, theta, part,
                        rnorm, c->st);
  else
    resid_launch<double>(c->n, c->rowptr.p, c->col.p, c->val.p, c->diag.p, X, k, k, theta, part,
                         rnorm, c->st);
}

}  // namespace vhci

using namespace vhci;

extern "C" vhci_status vhci_residual_norms(vhci_ctx* c, const double* X, const double* theta,
                                           double* rnorm, int k) {
  if (!c || !X || !theta || !rnorm || k <= 0) return VHCI_E_INPUT;
  if (is_sharded(c)) return fail(c, VHCI_E_STATE, "vhci_residual_norms on a sharded context");
  if (!c->h_valid || c->h_rows) VTRY(build_h(c, true));
  const int64_t n = c->n;
  std::vector<double> h((size_t)n * k);
  for (int64_t i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) h[(size_t)i * k + j] = X[(size_t)j * n + i];
  DBuf<double> dx, dth, part, dr;
  VCK(dx.reserve(h.size(), c->st));
  VCK(dth.reserve(k, c->st));
  VCK(part.reserve(resid_scratch_elems(k), c->st));
  VCK(dr.reserve(k, c->st));
  VCK(h2d(c, dx.p, h.data(), h.size() * sizeof(double)));
  VCK(h2d(c, dth.p, theta, k * sizeof(double)));
  residual_norms_fused(c, dx.p, k, dth.p, part.p, dr.p);
  VCK(d2h(c, rnorm, dr.p, k * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  VCK(cudaGetLastError());
  dx.release(c->st);
  dth.release(c->st);
  part.release(c->st);
  dr.release(c->st);
  return VHCI_OK;
}

// ---- residual norms without allocation ------------------------------------------------------
//
// Some callers cannot allocate device memory at the point where they need this check: a serving
// process whose device memory is owned by its own pool, or code that must not trigger the implicit
// device-wide synchronisation of cudaMalloc/cudaFree in the middle of its work.  For them the
// per-block partial sums live in a fixed array in the library's device memory instead of a buffer
// allocated per call.  The array holds kResidBlocks x kNoAllocMaxCols doubles (606 KB) and stays
// resident on every device that loads the library until the process exits.

namespace {

constexpr int kNoAllocMaxCols = 256;
__device__ __align__(256) double g_resid_scratch[kResidBlocks * kNoAllocMaxCols];

std::mutex g_scratch_mu;
double* g_scratch_dev[128] = {nullptr};  // device address of g_resid_scratch per device ordinal

// Restores the calling thread's current device on every return path.
struct DeviceGuard {
  int prev = -1;
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// True when p is device (or managed) memory that device `dev` can address.  Asks the runtime
// about the pointer; nothing is allocated.
bool device_pointer_on(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the (non-sticky) error an unknown pointer may leave
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" vhci_status vhci_residual_norms_noalloc(vhci_ctx* c, const double* X_dev,
                                                   const double* theta_dev, double* rnorm_dev,
                                                   int k) {
  if (!c || !X_dev || !theta_dev || !rnorm_dev) return VHCI_E_INPUT;
  if (k <= 0 || k > kNoAllocMaxCols)
    return fail(c, VHCI_E_INPUT,
                "vhci_residual_norms_noalloc: k must be between 1 and 256 (the size of its "
                "fixed scratch array)");
  if (!c->h_valid)
    return fail(c, VHCI_E_STATE,
                "vhci_residual_norms_noalloc: the Hamiltonian is not built; call vhci_build_h "
                "first (building it allocates, this call does not)");
  if (c->h_rows)
    return fail(c, VHCI_E_STATE, "vhci_residual_norms_noalloc: the Hamiltonian is sharded");
  const int dev = c->o.device;
  if (dev < 0 || dev >= 128) return fail(c, VHCI_E_CUDA, "device ordinal out of range");
  DeviceGuard guard;
  VCK(cudaGetDevice(&guard.prev));
  VCK(cudaSetDevice(dev));
  if (!device_pointer_on(X_dev, dev) || !device_pointer_on(theta_dev, dev) ||
      !device_pointer_on(rnorm_dev, dev))
    return fail(c, VHCI_E_INPUT,
                "vhci_residual_norms_noalloc: X_dev, theta_dev and rnorm_dev must be device "
                "memory of the context's device");
  double* scratch = nullptr;
  {
    // set-up, once per device with that device current: host code only has a host-side stand-in
    // for the array's name, so the device address is looked up and kept
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_resid_scratch);
      if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetSymbolAddress(g_resid_scratch)");
      g_scratch_dev[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_dev[dev];
  }
  // every block writes all of its partial sums, so nothing left from an earlier call is read
  residual_norms_fused(c, X_dev, k, theta_dev, scratch, rnorm_dev);
  VCK(cudaGetLastError());
  VCK(cudaStreamSynchronize(c->st));
  return VHCI_OK;
}
