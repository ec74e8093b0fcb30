// Host orchestration: Epstein-Nesbet PT2 (PT2.cpp:16-154), the heat-bath driver loop
// (Perform_HCI, HB.cpp:176-265; VHCI.cpp:49-80) and the reference's output and checkpoint files
// (PrintFreqs, Ham.cpp:448-502; Write/ReadCheckpoint, Core_functions.cpp:94-167).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <thread>

#include "internal.h"

namespace vhci {

int pt2(vhci_ctx* c, double eps2, double* dE_out, int64_t* n_pert) {
  if (c->nvec < 1 || c->x_rows != c->n) return fail(c, VHCI_E_STATE, "PT2 needs eigenvectors");
  cudaStream_t s = c->st;
  EventPair ev_t0t1;
  VCK(ev_t0t1.create());
  cudaEvent_t t0 = ev_t0t1.a, t1 = ev_t0t1.b;
  VCK(cudaEventRecord(t0, s));
  const int64_t n = c->n;
  const int nopt = (int)std::min<int64_t>(std::min<int64_t>(c->M.nstate, n), c->nvec);
  // perturber space: heat-bath screened states outside the basis (PT2.cpp:29-50)
  VTRY(generate_new_set(c, eps2));
  const int64_t np = c->nsel;
  if (c->o.max_pert > 0 && np > c->o.max_pert)
    return fail(c, VHCI_E_LIMIT, "perturber space of " + std::to_string(np) +
                                     " states exceeds max_pert " + std::to_string(c->o.max_pert));
  const KeyLayout L = c->L;
  std::vector<double> dE(nopt, 0.0);
  c->stats.pt2_perturbers += np;
  if (np > 0) {
    // perturber keys and hash
    DBuf<uint64_t> pkeys, pslots;
    VCK(pkeys.reserve((size_t)np * L.W, s));
    VCK(cudaMemcpyAsync(pkeys.p, c->sel.p, (size_t)np * L.W * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    uint64_t ns = 1024;
    while (ns < (uint64_t)(2 * np)) ns <<= 1;
    VCK(pslots.reserve(ns, s));
    hash_clear(pslots.p, ns, s);
    hash_insert_range(pslots.p, ns - 1, pkeys.p, 0, np, L.W, c->flags.p, s);
    HashView pv{pslots.p, ns - 1, pkeys.p};
    // this rank's perturbers [A0, A1): all of them, or one contiguous share on a sharded context
    // (the vectors are held whole on every rank, so each share is computed independently)
    const int R = is_sharded(c) ? c->comm.nranks : 1, rk = is_sharded(c) ? c->comm.rank : 0;
    const int64_t A0 = np * rk / R, A1 = np * (rk + 1) / R, NA = A1 - A0;
    // entry counts per perturber row (row a at index a - A0)
    DBuf<int32_t> acount;
    DBuf<int64_t> arow, tmp;
    VCK(acount.reserve(std::max<int64_t>(NA, 1), s));
    VCK(arow.reserve(NA + 1, s));
    VCK(tmp.reserve(std::max<int64_t>(scan_tmp_elems(NA), 1), s));
    VCK(cudaMemsetAsync(acount.p, 0, std::max<int64_t>(NA, 1) * sizeof(int32_t), s));
    pt2_count(c->keys.p, n, L, pv, conn_view(c), A0, A1, acount.p, s);
    exclusive_scan_i32(acount.p, arow.p, NA, tmp.p, s);
    int64_t total = 0;
    VCK(d2h(c, &total, arow.p + NA, sizeof(int64_t)));
    VCK(cudaStreamSynchronize(s));
    c->stats.pt2_entries += total;
    // chunk the perturber range so one chunk's entries fit the budget
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    // entries (12 bytes) plus, in the worst case, the same again as scratch for long-row ordering
    int64_t budget = c->o.pt2_chunk > 0 ? c->o.pt2_chunk : (int64_t)(freeb * 0.4 / 12.0);
    budget = std::max<int64_t>(budget, 1 << 20);
    // chunk bounds in perturber indices (arow_h is indexed from A0); one chunk needs only the total,
    // several the host copy of the row offsets
    std::vector<int64_t> bounds{A0};
    std::vector<int64_t> arow_h;
    if (total <= budget) {
      bounds.push_back(A1);
    } else {
      arow_h.resize(NA + 1);
      VCK(d2h(c, arow_h.data(), arow.p, (NA + 1) * sizeof(int64_t)));
      VCK(cudaStreamSynchronize(s));
    }
    auto chunk_entries = [&](int64_t a0, int64_t a1) {
      return arow_h.empty() ? total : arow_h[a1 - A0] - arow_h[a0 - A0];
    };
    while (bounds.back() < A1) {
      const int64_t a0 = bounds.back();
      const int64_t lim = arow_h[a0 - A0] + budget;
      int64_t a1 = A0 + (std::upper_bound(arow_h.begin() + (a0 - A0) + 1, arow_h.end(), lim) -
                         arow_h.begin()) - 1;
      if (a1 <= a0) a1 = a0 + 1;
      bounds.push_back(std::min(a1, A1));
    }
    DBuf<int32_t> ecol;
    DBuf<double> eval, part, dEd, Ed;
    const int64_t maxchunk = [&] {
      int64_t mx = 0;
      for (size_t q = 1; q < bounds.size(); ++q)
        mx = std::max(mx, chunk_entries(bounds[q - 1], bounds[q]));
      return mx;
    }();
    VCK(ecol.reserve(std::max<int64_t>(maxchunk, 1), s));
    VCK(eval.reserve(std::max<int64_t>(maxchunk, 1), s));
    const int nblk = pt2_en_blocks();
    VCK(part.reserve((size_t)nblk * nopt, s));
    VCK(cudaMemsetAsync(part.p, 0, (size_t)nblk * nopt * sizeof(double), s));
    VCK(dEd.reserve(nopt, s));
    VCK(Ed.reserve(nopt, s));
    VCK(cudaMemsetAsync(dEd.p, 0, nopt * sizeof(double), s));
    VCK(h2d(c, Ed.p, c->E.data(), nopt * sizeof(double)));
    DBuf<int64_t> crow, lrow_d, loff_d;
    DBuf<int32_t> lcol;
    DBuf<double> lval;
    DBuf<unsigned long long> lcnt;
    VCK(lcnt.reserve(2, s));
    for (size_t q = 1; q < bounds.size(); ++q) {
      const int64_t a0 = bounds[q - 1], a1 = bounds[q], na = a1 - a0;
      // this chunk's row offsets, rebased on the device
      VCK(crow.reserve(na + 1, s));
      pt2_rebase_rows(arow.p + (a0 - A0), na, crow.p, s);
      // rows too long for one warp's ordering, listed on the device; only their count and
      // entries come back, to size the scratch and the launch
      const int64_t maxlong = std::min<int64_t>(na, chunk_entries(a0, a1) / pt2_sort_long_min() + 1);
      VCK(lrow_d.reserve(std::max<int64_t>(maxlong, 1), s));
      VCK(loff_d.reserve(std::max<int64_t>(maxlong, 1), s));
      VCK(cudaMemsetAsync(lcnt.p, 0, 2 * sizeof(unsigned long long), s));
      pt2_list_long(crow.p, na, lrow_d.p, loff_d.p, lcnt.p, s);
      unsigned long long lc[2] = {0, 0};
      VCK(d2h(c, lc, lcnt.p, sizeof(lc)));
      VCK(cudaStreamSynchronize(s));
      VCK(cudaMemsetAsync(acount.p, 0, na * sizeof(int32_t), s));
      pt2_fill(c->keys.p, n, L, pv, conn_view(c), a0, a1, crow.p, acount.p, ecol.p, eval.p, s);
      // fixed entry order per row (the fill's atomics leave it arbitrary): short rows by one warp
      // each, long rows by one block each
      pt2_sort_rows(crow.p, na, ecol.p, eval.p, s);
      if (lc[0] > 0) {
        VCK(lcol.reserve((int64_t)lc[1], s));
        VCK(lval.reserve((int64_t)lc[1], s));
        for (int64_t q0 = 0; q0 < (int64_t)lc[0]; q0 += 65535)
          pt2_sort_long(crow.p, lrow_d.p + q0, loff_d.p + q0,
                        (int)std::min<int64_t>(65535, (int64_t)lc[0] - q0), ecol.p, eval.p, lcol.p,
                        lval.p, s);
      }
      EventPair ev_r0r1;
      VCK(ev_r0r1.create());
      cudaEvent_t r0 = ev_r0r1.a, r1 = ev_r0r1.b;
      VCK(cudaEventRecord(r0, s));
      if (!pt2_en(pkeys.p, a0, a1, L, conn_view(c), crow.p, ecol.p, eval.p, c->X.p, c->ldx, nopt,
                  Ed.p, part.p, s))
        return fail(c, VHCI_E_INPUT, "PT2: unsupported key width or state count");
      VCK(cudaEventRecord(r1, s));
      reduce_parts(part.p, nblk, nopt, dEd.p, s);
      VCK(cudaEventSynchronize(r1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, r0, r1);
      c->stats.ms_pt2_reduce += ms;
      const int64_t ent = chunk_entries(a0, a1);
      c->stats.pt2_reduce_bytes += ent * (4 + 8) + ent * (int64_t)nopt * 8 + (a1 - a0) * (8 + 8 * L.W);
    }
    VTRY(comm_sum(c, dEd.p, nopt));  // the ranks' shares of the perturber sum
    VCK(d2h(c, dE.data(), dEd.p, nopt * sizeof(double)));
    VCK(cudaStreamSynchronize(s));
    VCK(cudaGetLastError());
    int fl = 0;
    VTRY(read_flags(c, &fl));
    if (fl & kFlagTableFull) return fail(c, VHCI_E_TABLE_FULL, "perturber hash full");
    pkeys.release(s); pslots.release(s); acount.release(s); arow.release(s); tmp.release(s);
    ecol.release(s); eval.release(s); part.release(s); dEd.release(s); Ed.release(s); crow.release(s);
    lrow_d.release(s); loff_d.release(s); lcol.release(s); lval.release(s); lcnt.release(s);
  }
  for (int j = 0; j < nopt; ++j) {
    c->E[j] += dE[j];
    if (dE_out) dE_out[j] = dE[j];
  }
  VCK(cudaEventRecord(t1, s));
  VCK(cudaEventSynchronize(t1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  c->stats.ms_pt2 += ms;
  if (n_pert) *n_pert = np;
  return VHCI_OK;
}

}  // namespace vhci

using namespace vhci;

namespace {

// "% sparse" of the reference (Ham.cpp:341-342) counts its stored pattern, structural zeros
// included; with opts.structural_nnz (the CLI's default) that count is reproduced when the gate
// patterns are few enough, else the line uses the stored nonzero entries.
void print_sparse(vhci_ctx* c) {
  const double nn = (double)c->n;
  double stored = (double)(c->nnz + c->n);
  int64_t st = 0;
  if (c->o.structural_nnz && structural_available(c) && structural_count(c, &st) == VHCI_OK)
    stored = (double)st;
  std::cout << "The Hamiltonian is " << std::fixed << std::setprecision(2)
            << 100 * (1. - stored / (nn * nn)) << "% sparse." << std::endl;
}

int write_cp(vhci_ctx* c, const char* path) {
  if (!path) return VHCI_OK;
  if (c->o.verbose) { std::cout << " Writing checkpoint file..."; std::cout.flush(); }
  const int r = vhci_write_checkpoint(c, path);
  if (c->o.verbose) {
    if (r == VHCI_OK) std::cout << "done." << '\n' << std::endl;
    else std::cout << '\n' << " Error: checkpoint file could not be found or no name was given." << '\n' << std::endl;
  }
  return VHCI_OK;
}


// ---- checkpoint text: "%.17f " fields and integer quanta, formatted and parsed in parallel ----

int host_threads(vhci_ctx* c) {
  int t = c->o.host_threads > 0 ? c->o.host_threads : (int)std::thread::hardware_concurrency();
  return std::max(1, std::min(t, 64));
}

template <class F>
void parallel_for(int T, F&& f) {
  if (T <= 1) { f(0); return; }
  std::vector<std::thread> th;
  for (int t = 1; t < T; ++t) th.emplace_back([&f, t] { f(t); });
  f(0);
  for (auto& x : th) x.join();
}

// Appends the value as printf("%.17f ") prints it: std::to_chars in fixed notation is correctly
// rounded, as glibc's printf is, so the text is the same.
void append_fixed17(std::string& b, double v) {
  char tmp[400];
  const auto r = std::to_chars(tmp, tmp + sizeof tmp, v, std::chars_format::fixed, 17);
  b.append(tmp, r.ptr);
  b += ' ';
}

inline void skip_space(const char*& p, const char* end) {
  while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
}

template <class I>
bool next_int(const char*& p, const char* end, I& v) {
  skip_space(p, end);
  if (p < end && *p == '+') ++p;
  const auto r = std::from_chars(p, end, v);
  if (r.ec != std::errc()) return false;
  p = r.ptr;
  return true;
}

bool next_double(const char*& p, const char* end, double& v) {
  skip_space(p, end);
  if (p < end && *p == '+') ++p;
  const auto r = std::from_chars(p, end, v);
  if (r.ec != std::errc()) return false;
  p = r.ptr;
  return true;
}

// Read-only mapping of a whole file.
struct MappedFile {
  const char* data = nullptr;
  size_t size = 0;
  int fd = -1;
  bool open(const char* path) {
    fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size <= 0) return false;
    size = (size_t)st.st_size;
    void* m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m == MAP_FAILED) { size = 0; return false; }
    data = (const char*)m;
    return true;
  }
  ~MappedFile() {
    if (data) munmap((void*)data, size);
    if (fd >= 0) ::close(fd);
  }
};

}  // namespace

extern "C" {

vhci_status vhci_hci(vhci_ctx* c, const char* checkpoint_path, vhci_iter_cb cb, void* user) {
  if (!c) return VHCI_E_INPUT;
  const bool v = c->o.verbose != 0;
  const int k = c->M.nstate;
  EventPair ev_t0t1;
  VCK(ev_t0t1.create());
  cudaEvent_t t0 = ev_t0t1.a, t1 = ev_t0t1.b;
  VCK(cudaEventRecord(t0, c->st));
  if (c->M.eps1 == 0.0) {  // conventional VCI over the initial basis (VHCI.cpp:49-76)
    if (!c->restart || c->nvec == 0) {
      if (v) { std::cout << "Constructing the Vibrational CI Hamiltonian..."; std::cout.flush(); }
      VTRY(build_h(c));
      if (v) {
        print_sparse(c);
        if (k == 1) std::cout << "done." << "\n" << "\n" << "Solving for the ground state..." << "\n" << std::endl;
        else std::cout << "done." << "\n" << "\n" << "Solving for the lowest " << k << " eigenstates..." << "\n" << std::endl;
      }
      VTRY(eigs(c, k));
      if (c->n > 100000) write_cp(c, checkpoint_path);
    }
  } else {  // heat-bath iterations (HB.cpp:176-265)
    int iter = 1;
    if (!c->restart) {
      if (v) {
        std::cout << " Initial basis size is: " << c->n << "\n";
        std::cout << " Constructing Hamiltonian...";
      }
      VTRY(build_h(c));
      if (v) std::cout << " Diagonalizing..." << std::endl;
      const int guard = std::max(4, k / 10);
      VTRY(dense_eigs(c, k + guard));
      if (v) std::cout << std::fixed << std::setprecision(2) << " ZPE is: " << c->E[0] << "\n" << std::endl;
      if (cb) cb(user, 0, c->n, c->E[0]);
    }
    for (;;) {
      if (v) std::cout << " Performing HCI iteration: " << iter << std::endl;
      int64_t nnew = 0;
      VTRY(vhci_select(c, c->M.eps1, 0, &nnew));
      if (c->o.max_basis > 0 && (double)nnew / (double)c->n > 0.01 && c->n + nnew > c->o.max_basis)
        return fail(c, VHCI_E_LIMIT, "basis of " + std::to_string(c->n + nnew) +
                                         " states would exceed max_basis " +
                                         std::to_string(c->o.max_basis));
      if ((double)nnew / (double)c->n <= 0.01) {
        if (v) std::cout << " Basis converged after " << iter - 1 << " iterations and contains "
                         << c->n << " product states." << std::endl;
        break;
      }
      VTRY(append_keys(c, c->sel.p, c->nsel));
      if (v) {
        std::cout << " Basis size after iteration " << iter << " is: " << c->n << std::endl;
        std::cout << " Constructing Hamiltonian...";
        std::cout.flush();
      }
      ++iter;
      VTRY(build_h(c));
      if (v) {
        print_sparse(c);
        if (k == 1) std::cout << " Finding the ground state..." << std::endl;
        else std::cout << " Finding the first " << k << " eigenstates..." << std::endl;
      }
      VTRY(eigs(c, k));
      c->stats.hci_iterations += 1;
      if (v) std::cout << std::fixed << std::setprecision(2) << " ZPE is: " << c->E[0] << std::endl << std::endl;
      if (cb) cb(user, iter - 1, c->n, c->E[0]);
      if (c->n > 100000) write_cp(c, checkpoint_path);
    }
  }
  VCK(cudaEventRecord(t1, c->st));
  VCK(cudaEventSynchronize(t1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  c->stats.ms_total += ms;
  return VHCI_OK;
}

vhci_status vhci_pt2(vhci_ctx* c, double eps2, double* dE, int64_t* n_pert) {
  if (!c) return VHCI_E_INPUT;
  const bool v = c->o.verbose != 0;
  if (v) std::cout << " Finding connected states..." << std::endl;
  int64_t np = 0;
  const int r = pt2(c, eps2, dE, &np);
  if (r != VHCI_OK) return r;
  c->stats.ms_total += 0;
  if (v) {
    const int nopt = (int)std::min<int64_t>(c->M.nstate, c->n);
    std::cout << " Perturbative space contains " << np << " states." << std::endl;
    if (c->M.nstate == 1)
      std::cout << " Calculating the 2nd-order perturbative correction on the ground state energy" << std::endl;
    else
      std::cout << " Calculating the 2nd-order perturbative correction for on first " << nopt << " eigenvalues." << std::endl;
    std::cout << std::fixed << std::setprecision(2) << " New ZPE after PT2 correction is: " << c->E[0] << std::endl;
  }
  if (n_pert) *n_pert = np;
  return VHCI_OK;
}

// PrintFreqs (Ham.cpp:448-502): line 0 = E_0 and the assignments of every basis state whose
// |C_m0| >= max|C_0| / 2 (no separator between them); line n = E_n - E_0 with assignments
// separated by two spaces.  min(Nstate, #eigenvalues) lines.
vhci_status vhci_write_freqs(const vhci_ctx* c0, const char* path) {
  vhci_ctx* c = const_cast<vhci_ctx*>(c0);
  if (!c || !path) return VHCI_E_INPUT;
  const int held = (int)std::min<int64_t>((int64_t)c->E.size(), c->nvec);
  const int nf = std::min(c->M.nstate, held);
  if (nf < 1) return fail(c, VHCI_E_STATE, "no eigenpairs to print");
  const int64_t n = c->n;
  const int nm = c->M.nm;
  std::vector<uint8_t> q((size_t)n * nm);
  int64_t nn = 0;
  VTRY(vhci_get_basis(c, q.data(), n, &nn));
  std::vector<double> C((size_t)n * nf);
  VTRY(vhci_get_vectors(c, C.data(), nullptr, nf));
  std::ofstream out(path);
  if (!out.good()) return fail(c, VHCI_E_INPUT, "Error: Could not output file.");
  auto assign = [&](int64_t m, std::ostream& os) {
    int nmode = 0;
    for (int l = 0; l < nm; ++l) {
      const int qq = q[(size_t)m * nm + l];
      if (qq > 0) {
        if (nmode > 0) os << "+";
        os << qq << "w" << l;
        ++nmode;
      }
    }
  };
  for (int s = 0; s < nf; ++s) {
    const double* col = C.data() + (size_t)s * n;
    double mx = -INFINITY, mn = INFINITY;
    for (int64_t m = 0; m < n; ++m) { mx = std::max(mx, col[m]); mn = std::min(mn, col[m]); }
    const double maxcoeff = std::max(std::fabs(mx), std::fabs(mn));
    if (s == 0) out << std::fixed << std::setprecision(10) << c->E[0] << "   ";
    else out << std::fixed << std::setprecision(12) << c->E[s] - c->E[0] << "   ";
    int state = 0;
    for (int64_t m = 0; m < n; ++m) {
      if (std::fabs(col[m]) >= maxcoeff / 2) {
        if (s > 0 && state > 0) out << "  ";
        out << std::fixed << std::setprecision(2) << std::fabs(col[m]) << " (";
        assign(m, out);
        out << ")";
        ++state;
      }
    }
    out << '\n';
  }
  out.flush();
  return VHCI_OK;
}

// WriteCheckpoint (Core_functions.cpp:94-117): "N M NEig", then frequencies and eigenvalues,
// then one row per basis state: quanta followed by its coefficients, all reals "%.17f".
vhci_status vhci_write_checkpoint(const vhci_ctx* c0, const char* path) {
  vhci_ctx* c = const_cast<vhci_ctx*>(c0);
  if (!c || !path) return VHCI_E_INPUT;
  if (std::string(path) == "none") return fail(c, VHCI_E_INPUT, "no checkpoint name given");
  const int64_t n = c->n;
  const int nm = c->M.nm;
  const int nv = (int)std::min<int64_t>(std::min<int64_t>(c->nvec, c->M.nstate), n);
  std::vector<uint8_t> q((size_t)n * nm);
  int64_t nn = 0;
  VTRY(vhci_get_basis(c, q.data(), n, &nn));
  std::vector<double> C((size_t)n * std::max(nv, 1));
  if (nv > 0) VTRY(vhci_get_vectors(c, C.data(), nullptr, nv));
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(c, VHCI_E_INPUT, "checkpoint file could not be opened");
  std::string head = std::to_string(n) + " " + std::to_string(nm) + " " + std::to_string(c->M.nstate) + "\n";
  for (int j = 0; j < nm; ++j) append_fixed17(head, c->M.freq[j]);
  for (int j = 0; j < nv; ++j) append_fixed17(head, c->E[j]);
  head += '\n';
  std::fwrite(head.data(), 1, head.size(), f);
  // rows formatted in parallel chunks, written in order
  const int T = host_threads(c);
  const int64_t rows = std::max<int64_t>(256, (int64_t)(32e6 / (4.0 * nm + 24.0 * nv + 1.0)));
  std::vector<std::string> buf(T);
  bool ok = true;
  for (int64_t r0 = 0; r0 < n && ok; r0 += rows * T) {
    parallel_for(T, [&](int t) {
      std::string& b = buf[t];
      b.clear();
      const int64_t lo = r0 + t * rows, hi = std::min(n, lo + rows);
      for (int64_t i = lo; i < hi; ++i) {
        for (int j = 0; j < nm; ++j) {
          b += std::to_string((int)q[(size_t)i * nm + j]);
          b += ' ';
        }
        for (int j = 0; j < nv; ++j) append_fixed17(b, C[(size_t)j * n + i]);
        b += '\n';
      }
    });
    for (int t = 0; t < T && ok; ++t)
      ok = std::fwrite(buf[t].data(), 1, buf[t].size(), f) == buf[t].size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(c, VHCI_E_INPUT, "checkpoint file could not be written");
  return VHCI_OK;
}

// ReadCheckpoint (Core_functions.cpp:119-167): validates the mode count, Nstate and the
// frequencies (exact equality), then replaces the basis and the vectors.  The file is mapped and
// its rows parsed in parallel.
vhci_status vhci_read_checkpoint(vhci_ctx* c, const char* path) {
  if (!c || !path) return VHCI_E_INPUT;
  MappedFile mf;
  if (!mf.open(path)) return fail(c, VHCI_E_INPUT, "checkpoint file could not be opened");
  const char* p = mf.data;
  const char* end = mf.data + mf.size;
  long long nb = 0;
  int m = 0, ne = 0;
  if (!next_int(p, end, nb) || !next_int(p, end, m) || !next_int(p, end, ne) || nb <= 0)
    return fail(c, VHCI_E_INPUT, "Error: malformed checkpoint file.");
  if (m != c->M.nm) return fail(c, VHCI_E_INPUT, "Error: Checkpoint file contains wrong number of fundamental modes!");
  if (ne != c->M.nstate) return fail(c, VHCI_E_INPUT, "Error: Checkpoint file contains wrong number of eigenstates!");
  for (int i = 0; i < m; ++i) {
    double f = 0;
    if (!next_double(p, end, f) || f != c->M.freq[i])
      return fail(c, VHCI_E_INPUT, "Error: Checkpoint file contains wrong fundamental frequencies!");
  }
  std::vector<double> E(ne);
  for (int i = 0; i < ne; ++i)
    if (!next_double(p, end, E[i])) return fail(c, VHCI_E_INPUT, "Error: truncated checkpoint file.");
  // rows: one per line after the header lines; split the rest of the file among the threads at
  // line starts, count each part's lines, then parse every part into its rows
  while (p < end && *p != '\n') ++p;
  if (p < end) ++p;
  const int T = host_threads(c);
  std::vector<const char*> cut(T + 1);
  cut[0] = p;
  cut[T] = end;
  for (int t = 1; t < T; ++t) {
    const char* x = p + (end - p) * t / T;
    if (x < cut[t - 1]) x = cut[t - 1];
    while (x < end && x > p && x[-1] != '\n') ++x;
    cut[t] = x;
  }
  std::vector<int64_t> lines(T + 1, 0);
  parallel_for(T, [&](int t) {
    int64_t k = 0;
    for (const char* x = cut[t]; x < cut[t + 1]; ++x) k += *x == '\n';
    if (cut[t + 1] == end && cut[t + 1] > cut[t] && end[-1] != '\n') ++k;  // last line unterminated
    lines[t + 1] = k;
  });
  for (int t = 0; t < T; ++t) lines[t + 1] += lines[t];
  if (lines[T] < nb) return fail(c, VHCI_E_INPUT, "Error: truncated checkpoint file.");
  std::vector<uint8_t> q((size_t)nb * m);
  std::vector<double> C((size_t)nb * ne);
  std::vector<int> bad(T, 0);
  parallel_for(T, [&](int t) {
    const char* x = cut[t];
    const char* e = cut[t + 1];
    for (int64_t i = lines[t]; i < std::min<int64_t>(lines[t + 1], nb); ++i) {
      for (int j = 0; j < m; ++j) {
        long long qq = 0;
        if (!next_int(x, e, qq)) { bad[t] = 1; return; }
        if (qq < 0 || qq > 255) { bad[t] = 2; return; }
        q[(size_t)i * m + j] = (uint8_t)qq;
      }
      for (int j = 0; j < ne; ++j)
        if (!next_double(x, e, C[(size_t)j * nb + i])) { bad[t] = 1; return; }
      while (x < e && *x != '\n') ++x;
      if (x < e) ++x;
    }
  });
  for (int t = 0; t < T; ++t) {
    if (bad[t] == 2) return fail(c, VHCI_E_KEY_OVERFLOW, "checkpoint quanta out of range");
    if (bad[t]) return fail(c, VHCI_E_INPUT, "Error: truncated checkpoint file.");
  }
  VTRY(vhci_set_basis(c, q.data(), nb));
  VTRY(vhci_set_vectors(c, C.data(), E.data(), ne));
  c->restart = 1;
  return VHCI_OK;
}

}  // extern "C"
