// Library context: device buffers, library handles and the host model behind one vhci_ctx.
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <string>
#include <vector>

#include "model.h"
#include "ops.h"
#include "vhci_gpu.h"

namespace vhci {

// Stream-ordered device buffer that grows on demand.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;  // elements
  cudaError_t reserve(size_t n, cudaStream_t s, bool keep = false) {
    if (n <= cap && p) return cudaSuccess;
    size_t nc = n < 16 ? 16 : n;
    if (keep) nc = nc + nc / 2;
    T* q = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&q, nc * sizeof(T), s);
    if (e != cudaSuccess) return e;
    if (keep && p && cap) cudaMemcpyAsync(q, p, cap * sizeof(T), cudaMemcpyDeviceToDevice, s);
    if (p) cudaFreeAsync(p, s);
    p = q;
    cap = nc;
    return cudaSuccess;
  }
  void release(cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    cap = 0;
  }
  void swap(DBuf& o) {
    std::swap(p, o.p);
    std::swap(cap, o.cap);
  }
};

// A group set on the device (see upload_groups): records, packed key deltas, segment table.
struct DevGroups {
  DBuf<GroupDev> groups;
  DBuf<int64_t> wdelta;
  DBuf<uint64_t> lkey;
  DBuf<int32_t> lseg;
  uint32_t lmask = 0;
  int maxl = -1;
  int64_t ngroups = 0;
  void release(cudaStream_t s) {
    groups.release(s); wdelta.release(s); lkey.release(s); lseg.release(s);
  }
};

struct Status {
  int code = VHCI_OK;
  std::string msg;
};

}  // namespace vhci

struct vhci_ctx {
  vhci::Model M;
  vhci::ConnTables conn;
  std::vector<vhci::HBEntry> hbe;
  std::vector<int64_t> hbcum;
  vhci_opts o{};
  int restart = 0;

  cudaStream_t st = nullptr;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t sol = nullptr;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;

  vhci::KeyLayout L{};

  // basis (packed keys) and its hash
  int64_t n = 0;
  vhci::DBuf<uint64_t> keys;
  vhci::DBuf<uint64_t> hslots;
  uint64_t hmask = 0;

  // tables on device
  vhci::DBuf<vhci::GroupDev> groups;
  vhci::DBuf<int64_t> wdelta;
  // the reference's pair-gate patterns, for the structural entry count (built on first use)
  bool gate_built = false, gate_over = false;
  vhci::ConnTables gate;
  vhci::DevGroups gate_dev;
  vhci::DBuf<uint64_t> lkey;       // lowered-mode segment index (see ConnDev)
  vhci::DBuf<int32_t> lseg;
  uint32_t lmask = 0;
  int maxl = -1;
  vhci::DBuf<vhci::TermDev> terms, dterms;
  vhci::DBuf<double> T, freq;
  vhci::DBuf<vhci::HBDev> hbdev;
  vhci::DBuf<double> hbabs;
  vhci::DBuf<int64_t> hbcumd;

  // sharded solve (vhci_set_comm, comm.nranks > 1): when h_rows is set the held Hamiltonian is
  // the row block [row0, row0 + nrow) of the basis; every rank's block has rblk = ceil(n/nranks)
  // rows (the last may be shorter), the layout of the gathered vector blocks
  vhci_comm comm{};
  bool h_rows = false;
  int64_t row0 = 0, nrow = 0, rblk = 0;

  // Hamiltonian (off-diagonal CSR + FP64 diagonal)
  bool h_valid = false;
  int64_t nnz = 0;
  // the stored (whole, unsharded) matrix covers the first h_prefix states of the basis; states
  // appended since need only their own rows (incremental build)
  int64_t h_prefix = 0;
  vhci::DBuf<int32_t> rowcnt;
  vhci::DBuf<int64_t> rowptr;
  vhci::DBuf<int32_t> col;
  vhci::DBuf<double> val;
  vhci::DBuf<float> valf;
  vhci::DBuf<double> diag;
  // column panels of the off-diagonal entries (built with H when the gathered block outgrows L2)
  int npanel = 0;
  int64_t panel_cw = 0;
  vhci::DBuf<int64_t> prow;
  vhci::DBuf<int32_t> pcol;
  vhci::DBuf<double> pval;
  vhci::DBuf<float> pvalf;

  // eigenpairs: X is row-major x_rows x ldx, nvec columns valid
  int nvec = 0, ldx = 0;
  int64_t x_rows = 0;
  vhci::DBuf<double> X;
  std::vector<double> E;

  // last selection result (sorted keys)
  vhci::DBuf<uint64_t> sel;
  int64_t nsel = 0;

  // scratch
  vhci::DBuf<int> flags;
  vhci::DBuf<int64_t> i64a, i64b, scan_tmp;
  vhci::DBuf<double> d64a;
  vhci::DBuf<uint64_t> u64a, u64b;
  vhci::DBuf<uint8_t> u8a;
  vhci::DBuf<unsigned long long> ull;
  vhci::DBuf<double> solver_work;
  vhci::DBuf<int> solver_info;

  std::string err;
  vhci_stats stats{};
};
