// C ABI core: context lifetime, key layout, device tables, basis/vectors I/O, heat-bath
// selection and the Hamiltonian build.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "internal.h"

namespace vhci {

int fail(vhci_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(vhci_ctx* c, cudaError_t e, const char* where) {
  cudaGetLastError();
  const int code = (e == cudaErrorMemoryAllocation) ? VHCI_E_OOM : VHCI_E_CUDA;
  return fail(c, code, std::string(where) + ": " + cudaGetErrorString(e));
}

int blas_fail(vhci_ctx* c, int st, const char* where) {
  return fail(c, VHCI_E_CUDA, std::string(where) + ": library status " + std::to_string(st));
}

HashView basis_view(vhci_ctx* c) { return HashView{c->hslots.p, c->hmask, c->keys.p}; }

ConnDev conn_view(vhci_ctx* c) {
  ConnDev d;
  d.groups = c->groups.p;
  d.wdelta = c->wdelta.p;
  d.ngroups = (int64_t)c->conn.groups.size();
  d.terms = c->terms.p;
  d.dterms = c->dterms.p;
  d.ndterms = (int)c->conn.diag_terms.size();
  d.T = c->T.p;
  d.freq = c->freq.p;
  d.nm = c->M.nm;
  d.lkey = c->lkey.p;
  d.lseg = c->lseg.p;
  d.lmask = c->lmask;
  d.maxl = c->maxl;
  return d;
}

HBTable hb_view(vhci_ctx* c) {
  return HBTable{c->hbdev.p, c->hbabs.p, c->hbcumd.p, (int)c->hbe.size()};
}

float event_ms(vhci_ctx* c) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev_a, c->ev_b);
  return ms;
}

int read_flags(vhci_ctx* c, int* flags) {
  int h = 0;
  VCK(d2h(c, &h, c->flags.p, sizeof(int)));
  VCK(cudaMemsetAsync(c->flags.p, 0, sizeof(int), c->st));
  VCK(cudaStreamSynchronize(c->st));
  *flags = h;
  return VHCI_OK;
}

static KeyLayout make_layout(int nm, int bits) {
  KeyLayout L;
  L.bits = bits;
  L.mpw = 64 / bits;
  L.W = (nm + L.mpw - 1) / L.mpw;
  L.qmax = (1 << bits) - 1;
  return L;
}

template <class T>
static int upload(vhci_ctx* c, DBuf<T>& b, const std::vector<T>& h) {
  VCK(b.reserve(std::max<size_t>(h.size(), 1), c->st));
  if (!h.empty())
    VCK(h2d(c, b.p, h.data(), h.size() * sizeof(T)));
  return VHCI_OK;
}

// ---- stream and library handles, pooled per device ----------------------------------------
// Creating cuBLAS and cuSOLVER handles costs tens of milliseconds; a context borrows a set (stream
// + handles) from its device's pool and returns it, idle, on destroy, so a process that runs many
// solves creates each set once.  Concurrent contexts hold different sets.  Pooled sets live until
// the process exits.
namespace {
struct HandleSet {
  int device;
  int priority;
  cudaStream_t st;
  cublasHandle_t blas;
  cusolverDnHandle_t sol;
};
std::mutex g_handle_mu;
std::vector<HandleSet> g_handle_pool;
}  // namespace

// Stream priority of a context: the requested value clamped to the device's range.
static int clamped_priority(int want) {
  if (want == 0) return 0;
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) return 0;
  return std::max(greatest, std::min(least, want));
}

static int acquire_handles(vhci_ctx* c) {
  const int prio = clamped_priority(c->o.stream_priority);
  c->o.stream_priority = prio;
  {
    std::lock_guard<std::mutex> lk(g_handle_mu);
    for (size_t i = 0; i < g_handle_pool.size(); ++i)
      if (g_handle_pool[i].device == c->o.device && g_handle_pool[i].priority == prio) {
        c->st = g_handle_pool[i].st;
        c->blas = g_handle_pool[i].blas;
        c->sol = g_handle_pool[i].sol;
        g_handle_pool.erase(g_handle_pool.begin() + i);
        return VHCI_OK;
      }
  }
  VCK(cudaStreamCreateWithPriority(&c->st, cudaStreamNonBlocking, prio));
  VBL(cublasCreate(&c->blas));
  VBL(cublasSetStream(c->blas, c->st));
  VBL(cusolverDnCreate(&c->sol));
  VBL(cusolverDnSetStream(c->sol, c->st));
  return VHCI_OK;
}

static void release_handles(vhci_ctx* c) {
  if (!c->st || !c->blas || !c->sol) {  // a partly built set is not pooled
    if (c->blas) cublasDestroy(c->blas);
    if (c->sol) cusolverDnDestroy(c->sol);
    if (c->st) cudaStreamDestroy(c->st);
    return;
  }
  cudaStreamSynchronize(c->st);
  std::lock_guard<std::mutex> lk(g_handle_mu);
  g_handle_pool.push_back(HandleSet{c->o.device, c->o.stream_priority, c->st, c->blas, c->sol});
}

// Layout-dependent tables (packed key deltas, ladder factors) and the layout-free ones.
// Device form of a group set under the current key layout: group records, packed key deltas per
// word, and the lowered-mode segment table (open addressing on the segment keys, load <= 1/2).
static int upload_groups(vhci_ctx* c, const ConnTables& t, DevGroups& dg) {
  const KeyLayout& L = c->L;
  std::vector<GroupDev> g(t.groups.size());
  std::vector<int64_t> wd(t.groups.size() * L.W, 0);
  for (size_t u = 0; u < g.size(); ++u) {
    const Group& s = t.groups[u];
    GroupDev d{};
    d.tb = s.term_begin;
    d.te = s.term_end;
    d.nchg = (uint8_t)s.nchg;
    for (int k = 0; k < s.nchg; ++k) {
      d.mode[k] = (uint8_t)s.mode[k];
      d.delta[k] = (int8_t)s.delta[k];
      const int w = s.mode[k] / L.mpw;
      wd[u * L.W + w] += (int64_t)((uint64_t)(int64_t)s.delta[k] << ((s.mode[k] % L.mpw) * L.bits));
    }
    g[u] = d;
  }
  VTRY(upload(c, dg.groups, g));
  VTRY(upload(c, dg.wdelta, wd));
  const size_t nseg = t.seg_key.size();
  size_t P = 64;
  while (P < 2 * nseg) P <<= 1;
  std::vector<uint64_t> lk(P, 0);
  std::vector<int32_t> ls(2 * P, 0);
  for (size_t q = 0; q < nseg; ++q) {
    size_t h = mix64(t.seg_key[q]) & (P - 1);
    while (lk[h] != 0) h = (h + 1) & (P - 1);
    lk[h] = t.seg_key[q];
    ls[2 * h] = t.seg_begin[q];
    ls[2 * h + 1] = t.seg_begin[q + 1] - t.seg_begin[q];
  }
  VTRY(upload(c, dg.lkey, lk));
  VTRY(upload(c, dg.lseg, ls));
  dg.lmask = (uint32_t)(P - 1);
  dg.ngroups = (int64_t)t.groups.size();
  // the index covers up to 126 modes and 6 lowered modes (the key packs 7 bits per mode)
  dg.maxl = (c->M.nm <= 126 && t.max_lowered <= 6 && nseg > 0) ? t.max_lowered : -1;
  return VHCI_OK;
}

int upload_tables(vhci_ctx* c) {
  const KeyLayout& L = c->L;
  if (c->gate_built) VTRY(upload_groups(c, c->gate, c->gate_dev));  // re-packed for the layout
  std::vector<GroupDev> g(c->conn.groups.size());
  std::vector<int64_t> wd(c->conn.groups.size() * L.W, 0);
  for (size_t u = 0; u < g.size(); ++u) {
    const Group& s = c->conn.groups[u];
    GroupDev d{};
    d.tb = s.term_begin;
    d.te = s.term_end;
    d.nchg = (uint8_t)s.nchg;
    for (int k = 0; k < s.nchg; ++k) {
      d.mode[k] = (uint8_t)s.mode[k];
      d.delta[k] = (int8_t)s.delta[k];
      const int w = s.mode[k] / L.mpw;
      wd[u * L.W + w] += (int64_t)((uint64_t)(int64_t)s.delta[k] << ((s.mode[k] % L.mpw) * L.bits));
    }
    g[u] = d;
  }
  auto conv = [](const std::vector<Term>& in) {
    std::vector<TermDev> out(in.size());
    for (size_t i = 0; i < in.size(); ++i) {
      TermDev t{};
      t.fc = in[i].fc;
      t.nk = in[i].nk;
      for (int k = 0; k < kMaxOrder; ++k) {
        t.mode[k] = in[i].mode[k];
        t.pw[k] = in[i].pw[k];
        t.dl[k] = in[i].dl[k];
      }
      out[i] = t;
    }
    return out;
  };
  std::vector<double> T;
  ladder_table(L.qmax, T);
  std::vector<HBDev> hb(c->hbe.size());
  std::vector<double> habs(c->hbe.size());
  for (size_t i = 0; i < hb.size(); ++i) {
    HBDev d{};
    d.zero_idx = c->hbe[i].zero_idx;
    d.nk = (uint8_t)c->hbe[i].nk;
    for (int k = 0; k < c->hbe[i].nk; ++k) {
      d.mode[k] = (uint8_t)c->hbe[i].modes[k];
      d.pw[k] = (uint8_t)c->hbe[i].powers[k];
    }
    hb[i] = d;
    habs[i] = c->hbe[i].absfc;
  }
  VTRY(upload(c, c->groups, g));
  VTRY(upload(c, c->wdelta, wd));
  // lowered-mode segment index: open addressing on the segment keys, load <= 1/2
  {
    const ConnTables& t = c->conn;
    const size_t nseg = t.seg_key.size();
    size_t P = 64;
    while (P < 2 * nseg) P <<= 1;
    std::vector<uint64_t> lk(P, 0);
    std::vector<int32_t> ls(2 * P, 0);
    for (size_t q = 0; q < nseg; ++q) {
      size_t h = mix64(t.seg_key[q]) & (P - 1);
      while (lk[h] != 0) h = (h + 1) & (P - 1);
      lk[h] = t.seg_key[q];
      ls[2 * h] = t.seg_begin[q];
      ls[2 * h + 1] = t.seg_begin[q + 1] - t.seg_begin[q];
    }
    VTRY(upload(c, c->lkey, lk));
    VTRY(upload(c, c->lseg, ls));
    c->lmask = (uint32_t)(P - 1);
    // the index covers up to 126 modes and 6 lowered modes (the key packs 7 bits per mode)
    c->maxl = (c->M.nm <= 126 && t.max_lowered <= 6 && nseg > 0) ? t.max_lowered : -1;
  }
  VTRY(upload(c, c->terms, conv(c->conn.terms)));
  VTRY(upload(c, c->dterms, conv(c->conn.diag_terms)));
  VTRY(upload(c, c->T, T));
  VTRY(upload(c, c->freq, c->M.freq));
  VTRY(upload(c, c->hbdev, hb));
  VTRY(upload(c, c->hbabs, habs));
  VTRY(upload(c, c->hbcumd, c->hbcum));
  return VHCI_OK;
}

// Hash capacity for n_total keys at load <= 1/2; rebuilds the table when it grows.
int ensure_hash(vhci_ctx* c, int64_t n_total) {
  uint64_t need = 1024;
  while (need < (uint64_t)(2 * n_total)) need <<= 1;
  if (c->hmask + 1 >= need && c->hslots.p) return VHCI_OK;
  VCK(c->hslots.reserve(need, c->st));
  c->hmask = need - 1;
  hash_clear(c->hslots.p, need, c->st);
  hash_insert_range(c->hslots.p, c->hmask, c->keys.p, 0, c->n, c->L.W, c->flags.p, c->st);
  return VHCI_OK;
}

int append_keys(vhci_ctx* c, const uint64_t* dkeys, int64_t m) {
  if (m <= 0) return VHCI_OK;
  const int64_t n1 = c->n + m;
  if ((uint64_t)n1 >= 0xFFFFFFF0ull) return fail(c, VHCI_E_OOM, "basis exceeds 2^32 states");
  VCK(c->keys.reserve((size_t)n1 * c->L.W, c->st, true));
  VCK(cudaMemcpyAsync(c->keys.p + (size_t)c->n * c->L.W, dkeys, sizeof(uint64_t) * m * c->L.W,
                      cudaMemcpyDeviceToDevice, c->st));
  const int64_t n0 = c->n;
  c->n = n1;
  uint64_t need = 1024;
  while (need < (uint64_t)(2 * n1)) need <<= 1;
  if (c->hmask + 1 >= need) {
    hash_insert_range(c->hslots.p, c->hmask, c->keys.p, n0, n1, c->L.W, c->flags.p, c->st);
  } else {
    c->hmask = 0;
    VTRY(ensure_hash(c, n1));
  }
  c->h_valid = false;
  c->npanel = 0;
  return VHCI_OK;
}

// Re-encode every key with 8-bit mode fields (a state reached more than 15 quanta in a mode).
int promote_layout(vhci_ctx* c) {
  if (c->L.bits == 8) return fail(c, VHCI_E_KEY_OVERFLOW, "a state needs more than 255 quanta in one mode");
  const KeyLayout A = c->L, B = make_layout(c->M.nm, 8);
  if (B.W > 8) return fail(c, VHCI_E_INPUT, "too many modes for the 8-bit key layout (max 64)");
  DBuf<uint64_t> nk;
  VCK(nk.reserve(std::max<int64_t>(c->keys.cap / A.W * B.W, (int64_t)c->n * B.W + 16), c->st));
  repack_keys(c->keys.p, A, nk.p, B, c->n, c->M.nm, c->st);
  c->keys.release(c->st);
  c->keys = nk;
  if (c->nsel > 0 && c->sel.p) {
    DBuf<uint64_t> ns;
    VCK(ns.reserve((size_t)c->nsel * B.W, c->st));
    repack_keys(c->sel.p, A, ns.p, B, c->nsel, c->M.nm, c->st);
    c->sel.release(c->st);
    c->sel = ns;
  }
  c->L = B;
  VTRY(upload_tables(c));
  c->hmask = 0;
  VTRY(ensure_hash(c, c->n));
  return VHCI_OK;
}

// ------------------------------------------------------------------ heat-bath selection ----

int generate_new_set(vhci_ctx* c, double eps) {
  if (c->nvec < 1 || c->x_rows != c->n)
    return fail(c, VHCI_E_STATE, "selection needs eigenvectors over the current basis");
  const int64_t n = c->n;
  const int nopt = (int)std::min<int64_t>(std::min<int64_t>(c->M.nstate, n), c->nvec);
  VCK(c->d64a.reserve(n, c->st));
  VCK(c->i64a.reserve(n + 1, c->st));
  VCK(c->scan_tmp.reserve(std::max<int64_t>(scan_tmp_elems(n), 1), c->st));
  for (int attempt = 0; attempt < 3; ++attempt) {
    cmax_rows(c->X.p, n, c->ldx, nopt, c->d64a.p, c->st);
    select_count(c->d64a.p, n, hb_view(c), eps, c->i64a.p, c->st);
    exclusive_scan(c->i64a.p, c->i64a.p, n, c->scan_tmp.p, c->st);
    int64_t total = 0;
    VCK(d2h(c, &total, c->i64a.p + n, sizeof(int64_t)));
    VCK(cudaStreamSynchronize(c->st));
    c->stats.select_candidates += total;
    c->nsel = 0;
    if (total == 0) return VHCI_OK;
    // candidate capacity: grows on overflow, never beyond the work count
    int64_t cap = std::min<int64_t>(total, std::max<int64_t>(4 * n, 1 << 22));
    bool promoted = false;
    for (;;) {
      uint64_t slots = 1024;
      while (slots < (uint64_t)(2 * cap)) slots <<= 1;
      const int W = c->L.W;
      VCK(c->u64a.reserve((size_t)cap * W, c->st));
      VCK(c->u64b.reserve(slots, c->st));
      VCK(c->u8a.reserve(cap, c->st));
      VCK(c->ull.reserve(2, c->st));
      VCK(cudaMemsetAsync(c->u8a.p, 0, cap, c->st));
      VCK(cudaMemsetAsync(c->ull.p, 0, 2 * sizeof(unsigned long long), c->st));
      hash_clear(c->u64b.p, slots, c->st);
      NewSetView ns{c->u64b.p, slots - 1, c->u64a.p, c->u8a.p, c->ull.p, (uint64_t)cap, c->flags.p};
      select_generate(c->keys.p, n, c->i64a.p, total, hb_view(c), c->L, basis_view(c), ns, c->st);
      int fl = 0;
      VTRY(read_flags(c, &fl));
      if (fl & kFlagKeyOverflow) {
        VTRY(promote_layout(c));
        promoted = true;
        break;
      }
      if (fl & (kFlagCandOverflow | kFlagTableFull)) {
        if (cap >= total) return fail(c, VHCI_E_TABLE_FULL, "candidate set overflow");
        cap = std::min<int64_t>(total, cap * 4);
        continue;
      }
      unsigned long long ncand = 0;
      VCK(d2h(c, &ncand, c->ull.p, sizeof(ncand)));
      VCK(cudaStreamSynchronize(c->st));
      ncand = std::min<unsigned long long>(ncand, (unsigned long long)cap);
      VCK(c->sel.reserve((size_t)std::max<unsigned long long>(ncand, 1) * W, c->st));
      newset_compact(c->u64a.p, c->u8a.p, (int64_t)ncand, W, c->sel.p, c->ull.p + 1, c->st);
      unsigned long long m = 0;
      VCK(d2h(c, &m, c->ull.p + 1, sizeof(m)));
      VCK(cudaStreamSynchronize(c->st));
      c->nsel = (int64_t)m;
      if (m > 1) {
        VCK(c->u64b.reserve((size_t)m * W, c->st));
        VCK(c->scan_tmp.reserve(std::max<int64_t>(radix_hist_elems((int64_t)m), 1), c->st));
        radix_sort_keys(c->sel.p, c->u64b.p, (int64_t)m, W, c->L.bits * c->M.nm,
                        c->scan_tmp.p, c->st);
      }
      return VHCI_OK;
    }
    if (!promoted) break;
  }
  return fail(c, VHCI_E_KEY_OVERFLOW, "selection could not settle a key layout");
}

// --------------------------------------------------------------------- Hamiltonian build ----

double device_available(vhci_ctx* c) {
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  double avail = (double)freeb;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, c->o.device) == cudaSuccess) {
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used)
      avail += (double)(reserved - used);
  }
  return avail;
}

void spmm_h(vhci_ctx* c, const double* X, int ldx, int b, double* Y, int ldy) {
  const bool f = c->o.precision == 1;
  if (c->npanel > 0)
    spmm_panels(c->nrow, c->npanel, c->prow.p, c->pcol.p, f ? nullptr : c->pval.p,
                f ? c->pvalf.p : nullptr, c->diag.p, X, ldx, b, Y, ldy, c->row0, c->st);
  else
    spmm(c->nrow, c->rowptr.p, c->col.p, f ? nullptr : c->val.p, f ? c->valf.p : nullptr,
         c->diag.p, X, ldx, b, Y, ldy, c->row0, c->st);
}

// Column panels for the product: one 16-column FP64 block row is 128 bytes, and each panel's rows
// take about 96 MB of the 126 MB L2, so panels start at two when the block's rows exceed 96 MB
// (N > 750k).  VHCI_PANEL_MB sets the panel size; VHCI_PANELS=0 turns panels off.  On the 6.1M-state, 1.17e9-entry matrix
// 96 MB panels measured 3 % faster than one pass and 48 MB ones no faster: the product there is
// bound by the dependent index-then-gather loads more than by where the block rows live.  Skipped when the regrouped copy does not fit
// in free device memory.
static int build_panels(vhci_ctx* c) {
  c->npanel = 0;
  const int64_t n = c->n;      // columns
  const int64_t nr = c->nrow;  // rows held
  if (const char* e = std::getenv("VHCI_PANELS"))
    if (std::atoi(e) == 0) return VHCI_OK;
  double pbytes = 96e6;
  if (const char* e = std::getenv("VHCI_PANEL_MB")) pbytes = std::max(0.01, std::atof(e)) * 1e6;
  int P = (int)std::ceil((double)n * 128.0 / pbytes);
  if (P < 2 || c->nnz == 0) return VHCI_OK;
  P = std::min(P, kMaxPanels);
  const int64_t cw = (n + P - 1) / P;
  P = (int)((n + cw - 1) / cw);
  const int64_t pn = (int64_t)P * nr;
  const double sval = c->o.precision == 1 ? 4.0 : 8.0;
  const double need = (double)c->nnz * (4.0 + sval) + (pn + 1) * 8.0 + pn * 4.0 +
                      scan_tmp_elems(pn) * 8.0 + 2e9;
  // the eigensolver's smallest working set must still fit after the panels: the panels are an
  // optimisation, the Lanczos basis is not
  if (need + lanczos_min_bytes(c, c->M.nstate) > device_available(c)) return VHCI_OK;
  DBuf<int32_t> cnt;
  DBuf<int64_t> tmp;
  VCK(cnt.reserve(pn, c->st));
  VCK(cudaMemsetAsync(cnt.p, 0, pn * sizeof(int32_t), c->st));
  panel_count(nr, c->rowptr.p, c->col.p, cw, cnt.p, c->st);
  VCK(c->prow.reserve(pn + 1, c->st));
  VCK(tmp.reserve(std::max<int64_t>(scan_tmp_elems(pn), 1), c->st));
  exclusive_scan_i32(cnt.p, c->prow.p, pn, tmp.p, c->st);
  VCK(c->pcol.reserve(c->nnz, c->st));
  if (c->o.precision == 1) VCK(c->pvalf.reserve(c->nnz, c->st));
  else VCK(c->pval.reserve(c->nnz, c->st));
  panel_fill(nr, c->rowptr.p, c->col.p, c->o.precision == 1 ? nullptr : c->val.p,
             c->o.precision == 1 ? c->valf.p : nullptr, cw, P, c->prow.p, c->pcol.p, c->pval.p,
             c->pvalf.p, c->st);
  cnt.release(c->st);
  tmp.release(c->st);
  VCK(cudaGetLastError());
  c->npanel = P;
  c->panel_cw = cw;
  return VHCI_OK;
}

// Entries of the reference's stored Hamiltonian pattern (Ham.cpp:236-344): the diagonal plus every
// ordered pair of basis states whose quanta differ by an admitted change (|delta|_1 = s, s even
// <= fcmax, s odd <= fcmax - 1), connected by a force constant or not (structural zeros).  The
// gate patterns are built once and walked with the Hamiltonian build's count pass.
constexpr int64_t kMaxGatePatterns = 2000000;

bool structural_available(vhci_ctx* c) {
  if (!c->gate_built && !c->gate_over) {
    if (build_gate_patterns(c->M, c->gate, kMaxGatePatterns)) {
      if (upload_groups(c, c->gate, c->gate_dev) != VHCI_OK) return false;
      c->gate_built = true;
    } else {
      c->gate_over = true;
    }
  }
  return c->gate_built;
}

int structural_count(vhci_ctx* c, int64_t* out) {
  const int64_t n = c->n;
  if (!structural_available(c))
    return fail(c, VHCI_E_LIMIT, "the pair gates admit more than " +
                                     std::to_string(kMaxGatePatterns) + " change patterns");
  ConnDev d = conn_view(c);
  d.groups = c->gate_dev.groups.p;
  d.wdelta = c->gate_dev.wdelta.p;
  d.ngroups = c->gate_dev.ngroups;
  d.lkey = c->gate_dev.lkey.p;
  d.lseg = c->gate_dev.lseg.p;
  d.lmask = c->gate_dev.lmask;
  d.maxl = c->gate_dev.maxl;
  DBuf<int64_t> sum;
  VCK(c->rowcnt.reserve(n, c->st));
  VCK(sum.reserve(n + 1, c->st));
  VCK(c->scan_tmp.reserve(std::max<int64_t>(scan_tmp_elems(n), 1), c->st));
  hbuild_count(c->keys.p, 0, n, c->L, basis_view(c), d, c->rowcnt.p, c->st);
  exclusive_scan_i32(c->rowcnt.p, sum.p, n, c->scan_tmp.p, c->st);
  int64_t pairs = 0;
  VCK(d2h(c, &pairs, sum.p + n, sizeof(int64_t)));
  VCK(cudaStreamSynchronize(c->st));
  sum.release(c->st);
  *out = n + pairs;
  return VHCI_OK;
}

// ---- collectives of a sharded solve ---------------------------------------------------------
// The callbacks run the caller's collectives on device buffers; the stream is synchronised first
// so the buffers hold their final values, and the callback completes the collective before it
// returns.

int comm_sum(vhci_ctx* c, double* buf, int64_t count) {
  if (!is_sharded(c) || count <= 0) return VHCI_OK;
  VCK(cudaStreamSynchronize(c->st));
  if (c->comm.allreduce_sum(c->comm.user, buf, count) != 0)
    return fail(c, VHCI_E_CUDA, "all-reduce of the sharded solve failed");
  return VHCI_OK;
}

int comm_gather(vhci_ctx* c, const void* send, void* recv, int64_t bytes) {
  if (!is_sharded(c)) {
    if (recv != send && bytes > 0)
      VCK(cudaMemcpyAsync(recv, send, bytes, cudaMemcpyDeviceToDevice, c->st));
    return VHCI_OK;
  }
  VCK(cudaStreamSynchronize(c->st));
  if (c->comm.allgather(c->comm.user, send, recv, bytes) != 0)
    return fail(c, VHCI_E_CUDA, "all-gather of the sharded solve failed");
  return VHCI_OK;
}

int comm_bcast0(vhci_ctx* c, double* buf, int64_t count) {
  if (!is_sharded(c) || count <= 0) return VHCI_OK;
  if (c->comm.rank != 0) VCK(cudaMemsetAsync(buf, 0, count * sizeof(double), c->st));
  return comm_sum(c, buf, count);
}

bool dense_path(int64_t n, int k) {
  const int guard = std::max(4, k / 10);
  const int64_t kk = std::min<int64_t>(n, k + guard);
  return n <= 2000 || n <= 3 * kk + 64;
}

// Incremental build: rows of the states appended since the stored matrix was built (states
// h_prefix .. n - 1), their entries in old columns transposed into the tails of the old rows
// (H is symmetric to the bit: each element's ladder factors come from the lower state), merged
// into a new CSR.  The transposed entries are radix-sorted by (column, entry), so each old row's
// tail lists its new columns in ascending order and the layout is the same on every run.
// Returns VHCI_OK, 1 when it declines (too many entries for the 32-bit entry keys, or not enough
// device memory to hold the old and the new matrix at once: the caller builds from scratch),
// or an error.
static int build_h_incremental(vhci_ctx* c) {
  const int64_t n = c->n, n_old = c->h_prefix, nn = n - n_old;
  cudaStream_t s = c->st;
  const bool f = c->o.precision == 1;
  const double vb = f ? 4.0 : 8.0;
  VCK(cudaEventRecord(c->ev_a, s));
  DBuf<int32_t> cnt_new, tcol, add, erow, len, col_all;
  DBuf<int64_t> rp_new, xoff, rp_all, hist;
  DBuf<double> tval, tdiag, val_all, diag_all;
  DBuf<float> tvalf, valf_all;
  DBuf<uint64_t> keys, alt;
  DBuf<unsigned long long> kc;
  auto release_all = [&] {
    cnt_new.release(s); tcol.release(s); add.release(s); erow.release(s); len.release(s);
    col_all.release(s); rp_new.release(s); xoff.release(s); rp_all.release(s); hist.release(s);
    tval.release(s); tdiag.release(s); val_all.release(s); diag_all.release(s); tvalf.release(s);
    valf_all.release(s); keys.release(s); alt.release(s); kc.release(s);
  };
  VCK(cnt_new.reserve(nn, s));
  VCK(rp_new.reserve(nn + 1, s));
  VCK(c->scan_tmp.reserve(std::max<int64_t>(scan_tmp_elems(n), 1), s));
  hbuild_count(c->keys.p, n_old, nn, c->L, basis_view(c), conn_view(c), cnt_new.p, s);
  exclusive_scan_i32(cnt_new.p, rp_new.p, nn, c->scan_tmp.p, s);
  int64_t nnz_new = 0;
  VCK(d2h(c, &nnz_new, rp_new.p + nn, sizeof(int64_t)));
  VCK(cudaStreamSynchronize(s));
  // working set: the new rows, their transposed keys (sorted through a second buffer), the entry
  // rows, and the merged matrix (at most nnz_old + 2 nnz_new entries) beside the stored one
  const double nnz_all_max = (double)c->nnz + 2.0 * (double)nnz_new;
  const double need = (double)nnz_new * (4.0 + vb + 16.0 + 4.0) + nnz_all_max * (4.0 + vb) +
                      (double)n * 40.0 + 8.0 * radix_hist_elems(nnz_new);
  const double eig = lanczos_min_bytes(c, c->M.nstate);
  const double old_bytes = (double)c->nnz * (4.0 + vb) + 16.0 * (double)n_old;
  const double avail = device_available(c);
  if (nnz_new >= 0xFFFFFFFFll || need > 0.9 * avail || nnz_all_max * (4.0 + vb) + eig > avail + old_bytes) {
    release_all();
    return 1;
  }
  VCK(tcol.reserve(std::max<int64_t>(nnz_new, 1), s));
  if (f) VCK(tvalf.reserve(std::max<int64_t>(nnz_new, 1), s));
  else VCK(tval.reserve(std::max<int64_t>(nnz_new, 1), s));
  VCK(tdiag.reserve(nn, s));
  hbuild_fill(c->keys.p, n_old, nn, c->L, basis_view(c), conn_view(c), rp_new.p, tcol.p,
              f ? nullptr : tval.p, f ? tvalf.p : nullptr, tdiag.p, s);
  // transposed entries: per old column counts and (column, entry) keys, sorted
  VCK(add.reserve(n_old, s));
  VCK(cudaMemsetAsync(add.p, 0, n_old * sizeof(int32_t), s));
  VCK(keys.reserve(std::max<int64_t>(nnz_new, 1), s));
  VCK(kc.reserve(1, s));
  VCK(cudaMemsetAsync(kc.p, 0, sizeof(unsigned long long), s));
  hmerge_cross_keys(tcol.p, nnz_new, n_old, add.p, keys.p, kc.p, s);
  unsigned long long ncross_u = 0;
  VCK(d2h(c, &ncross_u, kc.p, sizeof(ncross_u)));
  VCK(cudaStreamSynchronize(s));
  const int64_t ncross = (int64_t)ncross_u;
  if (ncross > 0) {
    int cbits = 1;
    while (cbits < 32 && ((int64_t)1 << cbits) < n_old) ++cbits;
    VCK(alt.reserve(ncross, s));
    VCK(hist.reserve(std::max<int64_t>(radix_hist_elems(ncross), 1), s));
    radix_sort_keys(keys.p, alt.p, ncross, 1, 32 + cbits, hist.p, s);
  }
  VCK(xoff.reserve(n_old + 1, s));
  exclusive_scan_i32(add.p, xoff.p, n_old, c->scan_tmp.p, s);
  VCK(erow.reserve(std::max<int64_t>(nnz_new, 1), s));
  hmerge_entry_rows(rp_new.p, nn, erow.p, s);
  // merged row pointers and arrays
  VCK(len.reserve(n, s));
  hmerge_lengths(c->rowptr.p, add.p, rp_new.p, n_old, nn, len.p, s);
  VCK(rp_all.reserve(n + 1, s));
  exclusive_scan_i32(len.p, rp_all.p, n, c->scan_tmp.p, s);
  const int64_t nnz_all = c->nnz + nnz_new + ncross;
  VCK(col_all.reserve(std::max<int64_t>(nnz_all, 1), s));
  if (f) VCK(valf_all.reserve(std::max<int64_t>(nnz_all, 1), s));
  else VCK(val_all.reserve(std::max<int64_t>(nnz_all, 1), s));
  VCK(diag_all.reserve(n, s));
  hmerge_copy_rows(c->rowptr.p, c->col.p, f ? nullptr : c->val.p, f ? c->valf.p : nullptr, n_old,
                   rp_all.p, col_all.p, val_all.p, valf_all.p, s);
  hmerge_copy_rows(rp_new.p, tcol.p, f ? nullptr : tval.p, f ? tvalf.p : nullptr, nn,
                   rp_all.p + n_old, col_all.p, val_all.p, valf_all.p, s);
  hmerge_cross_scatter(keys.p, ncross, xoff.p, c->rowptr.p, rp_all.p, erow.p,
                       f ? nullptr : tval.p, f ? tvalf.p : nullptr, n_old, col_all.p, val_all.p,
                       valf_all.p, s);
  VCK(cudaMemcpyAsync(diag_all.p, c->diag.p, n_old * sizeof(double), cudaMemcpyDeviceToDevice, s));
  VCK(cudaMemcpyAsync(diag_all.p + n_old, tdiag.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // the merged matrix replaces the stored one (the old arrays leave with the temporaries)
  std::swap(c->rowptr.p, rp_all.p); std::swap(c->rowptr.cap, rp_all.cap);
  std::swap(c->col.p, col_all.p); std::swap(c->col.cap, col_all.cap);
  if (f) { std::swap(c->valf.p, valf_all.p); std::swap(c->valf.cap, valf_all.cap); }
  else { std::swap(c->val.p, val_all.p); std::swap(c->val.cap, val_all.cap); }
  std::swap(c->diag.p, diag_all.p); std::swap(c->diag.cap, diag_all.cap);
  release_all();
  c->nnz = nnz_all;
  c->row0 = 0;
  c->nrow = n;
  c->rblk = n;
  VTRY(build_panels(c));
  VCK(cudaEventRecord(c->ev_b, s));
  VCK(cudaEventSynchronize(c->ev_b));
  VCK(cudaGetLastError());
  c->stats.ms_hbuild += event_ms(c);
  c->stats.hbuild_probes += 2 * nn * (int64_t)c->conn.groups.size();
  c->stats.hbuild_incremental += 1;
  c->h_prefix = n;
  c->h_valid = true;
  return VHCI_OK;
}

int build_h(vhci_ctx* c, bool all_rows) {
  const int64_t n = c->n;
  c->npanel = 0;
  c->pcol.release(c->st);  // the previous panels: freed before the new matrix is built
  c->pval.release(c->st);
  c->pvalf.release(c->st);
  c->prow.release(c->st);
  // rows held: every row, or this rank's block when the solve is sharded and sparse
  c->h_rows = !all_rows && is_sharded(c) && !dense_path(n, c->M.nstate);
  if (c->h_rows) {
    c->rblk = (n + c->comm.nranks - 1) / c->comm.nranks;
    c->row0 = std::min<int64_t>(n, (int64_t)c->comm.rank * c->rblk);
    c->nrow = std::min<int64_t>(c->rblk, n - c->row0);
  } else {
    c->row0 = 0;
    c->nrow = n;
    c->rblk = n;
  }
  const int64_t r0 = c->row0, nr = c->nrow;
  if (!c->h_rows && c->h_prefix > 0 && c->h_prefix < n) {
    const int r = build_h_incremental(c);
    if (r != 1) return r;
  }
  c->h_prefix = 0;
  VCK(cudaEventRecord(c->ev_a, c->st));
  VCK(c->rowcnt.reserve(std::max<int64_t>(nr, 1), c->st));
  VCK(c->rowptr.reserve(nr + 1, c->st));
  VCK(c->scan_tmp.reserve(std::max<int64_t>(scan_tmp_elems(nr), 1), c->st));
  hbuild_count(c->keys.p, r0, nr, c->L, basis_view(c), conn_view(c), c->rowcnt.p, c->st);
  exclusive_scan_i32(c->rowcnt.p, c->rowptr.p, nr, c->scan_tmp.p, c->st);
  int64_t nnz = 0;
  VCK(d2h(c, &nnz, c->rowptr.p + nr, sizeof(int64_t)));
  VCK(cudaStreamSynchronize(c->st));
  // the previous matrix's arrays are replaced, not grown in place: release them first so the old
  // and new matrix never coexist
  if ((int64_t)c->col.cap < nnz) c->col.release(c->st);
  if ((int64_t)c->val.cap < nnz) c->val.release(c->st);
  if ((int64_t)c->valf.cap < nnz) c->valf.release(c->st);
  {  // admission: the matrix and the eigensolver's smallest working set must fit together
    const double hbytes = (double)nnz * (4.0 + (c->o.precision == 1 ? 4.0 : 8.0)) + 8.0 * nr;
    const double avail = device_available(c) + 8.0 * (double)c->x_rows * c->ldx;
    const double eig = lanczos_min_bytes(c, c->M.nstate);
    if (hbytes + eig > avail) {
      char msg[320];
      std::snprintf(msg, sizeof msg,
                    "Hamiltonian rows of %lld states and %lld off-diagonal entries need %.1f GB "
                    "(plus %.1f GB for the eigensolver); %.1f GB of device memory is available",
                    (long long)nr, (long long)nnz, hbytes / 1e9, eig / 1e9, avail / 1e9);
      return fail(c, VHCI_E_OOM, msg);
    }
  }
  VCK(c->col.reserve(std::max<int64_t>(nnz, 1), c->st));
  if (c->o.precision == 1) {
    VCK(c->valf.reserve(std::max<int64_t>(nnz, 1), c->st));
  } else {
    VCK(c->val.reserve(std::max<int64_t>(nnz, 1), c->st));
  }
  VCK(c->diag.reserve(std::max<int64_t>(nr, 1), c->st));
  hbuild_fill(c->keys.p, r0, nr, c->L, basis_view(c), conn_view(c), c->rowptr.p, c->col.p,
              c->o.precision == 1 ? nullptr : c->val.p, c->o.precision == 1 ? c->valf.p : nullptr,
              c->diag.p, c->st);
  c->nnz = nnz;
  VTRY(build_panels(c));
  VCK(cudaEventRecord(c->ev_b, c->st));
  VCK(cudaEventSynchronize(c->ev_b));
  VCK(cudaGetLastError());
  c->stats.ms_hbuild += event_ms(c);
  c->stats.hbuild_probes += 2 * nr * (int64_t)c->conn.groups.size();
  c->nnz = nnz;
  c->h_valid = true;
  c->h_prefix = c->h_rows ? 0 : n;
  return VHCI_OK;
}

static int create_common(vhci_ctx* c, int restart) {
  std::string err;
  if (!finalize_model(c->M, restart != 0, err)) return fail(c, VHCI_E_INPUT, err);
  build_conn_tables(c->M, c->conn);
  build_hb_entries(c->M, c->hbe, c->hbcum);
  int maxq = 0;
  for (uint8_t q : c->M.init_basis) maxq = std::max<int>(maxq, q);
  c->L = make_layout(c->M.nm, maxq > 15 ? 8 : 4);
  if (c->L.W > 8 && c->L.bits == 4) return fail(c, VHCI_E_INPUT, "too many modes (max 128)");
  if (c->L.W > 8) return fail(c, VHCI_E_INPUT, "too many modes for the 8-bit key layout (max 64)");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(c, VHCI_E_CUDA, "no CUDA device available (this library has no CPU path)");
  if (c->o.device < 0 || c->o.device >= ndev) return fail(c, VHCI_E_CUDA, "bad device ordinal");
  VCK(cudaSetDevice(c->o.device));
  VCK(cudaEventCreate(&c->ev_a));
  VCK(cudaEventCreate(&c->ev_b));
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, c->o.device) == cudaSuccess) {
      uint64_t thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  VTRY(acquire_handles(c));
  VCK(c->flags.reserve(4, c->st));
  VCK(cudaMemsetAsync(c->flags.p, 0, 4 * sizeof(int), c->st));
  VTRY(upload_tables(c));
  // initial basis
  const int64_t n0 = c->M.n0;
  DBuf<uint8_t> q;
  VCK(q.reserve(std::max<int64_t>(n0 * c->M.nm, 1), c->st));
  VCK(h2d(c, q.p, c->M.init_basis.data(), n0 * c->M.nm));
  VCK(c->keys.reserve((size_t)std::max<int64_t>(n0, 16) * c->L.W, c->st));
  pack_keys(q.p, n0, c->M.nm, c->L, c->keys.p, c->st);
  q.release(c->st);
  c->n = n0;
  c->hmask = 0;
  VTRY(ensure_hash(c, n0));
  int fl = 0;
  VTRY(read_flags(c, &fl));
  if (fl) return fail(c, VHCI_E_INPUT, "duplicate states in the initial basis");
  c->restart = restart;
  return VHCI_OK;
}

}  // namespace vhci

using namespace vhci;

extern "C" {

void vhci_default_opts(vhci_opts* o) {
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->precision = 0;
  o->eig_tol = 1e-10;
  o->eig_maxit = 1000;
  o->verbose = 0;
  o->host_threads = 1;
  o->pt2_chunk = 0;
  o->structural_nnz = 0;
}

vhci_status vhci_create_from_file(const char* path, const vhci_opts* o, int restart,
                                  vhci_ctx** out) {
  if (!out) return VHCI_E_INPUT;
  *out = nullptr;
  vhci_ctx* c = new vhci_ctx();
  if (o) c->o = *o; else vhci_default_opts(&c->o);
  std::string err;
  int r = VHCI_OK;
  if (!parse_input_file(path, c->M, err)) r = fail(c, VHCI_E_INPUT, err);
  else r = create_common(c, restart);
  *out = c;  // returned even on failure so vhci_last_error() can report; caller destroys
  return r;
}

vhci_status vhci_create(const vhci_problem* p, const vhci_opts* o, int restart, vhci_ctx** out) {
  if (!out) return VHCI_E_INPUT;
  *out = nullptr;
  vhci_ctx* c = new vhci_ctx();
  if (o) c->o = *o; else vhci_default_opts(&c->o);
  std::string err;
  int r = VHCI_OK;
  if (!model_from_problem(p, c->M, err)) r = fail(c, VHCI_E_INPUT, err);
  else r = create_common(c, restart);
  *out = c;
  return r;
}

vhci_status vhci_destroy(vhci_ctx* c) {
  if (!c) return VHCI_OK;
  if (c->st) {
    cudaStreamSynchronize(c->st);
    c->keys.release(c->st); c->hslots.release(c->st);
    c->groups.release(c->st); c->wdelta.release(c->st); c->terms.release(c->st);
    c->dterms.release(c->st); c->T.release(c->st); c->freq.release(c->st);
    c->hbdev.release(c->st); c->hbabs.release(c->st); c->hbcumd.release(c->st);
    c->rowcnt.release(c->st); c->rowptr.release(c->st); c->col.release(c->st);
    c->val.release(c->st); c->valf.release(c->st); c->diag.release(c->st);
    c->X.release(c->st); c->sel.release(c->st); c->flags.release(c->st);
    c->i64a.release(c->st); c->i64b.release(c->st); c->scan_tmp.release(c->st);
    c->d64a.release(c->st); c->u64a.release(c->st); c->u64b.release(c->st);
    c->u8a.release(c->st); c->ull.release(c->st); c->solver_work.release(c->st);
    c->solver_info.release(c->st);
    c->lkey.release(c->st); c->lseg.release(c->st);
    c->prow.release(c->st); c->pcol.release(c->st); c->pval.release(c->st);
    c->pvalf.release(c->st); c->gate_dev.release(c->st);
    cudaStreamSynchronize(c->st);
  }
  if (c->ev_a) cudaEventDestroy(c->ev_a);
  if (c->ev_b) cudaEventDestroy(c->ev_b);
  release_handles(c);
  delete c;
  return VHCI_OK;
}

vhci_status vhci_last_error(const vhci_ctx* c, char* buf, size_t n) {
  if (!c || !buf || n == 0) return VHCI_E_INPUT;
  std::snprintf(buf, n, "%s", c->err.c_str());
  return VHCI_OK;
}

vhci_status vhci_get_info(const vhci_ctx* c, vhci_info* info) {
  if (!c || !info) return VHCI_E_INPUT;
  info->nmodes = c->M.nm;
  info->nstate = c->M.nstate;
  info->pt2 = c->M.pt2;
  info->key_bits = c->L.bits;
  info->key_words = c->L.W;
  info->eps1 = c->M.eps1;
  info->eps2 = c->M.eps2;
  info->n_basis = c->n;
  info->n_fc = (int64_t)c->M.fcs.size();
  info->n_hb = (int64_t)c->M.hb.size();
  info->n_groups = (int64_t)c->conn.groups.size();
  info->n_vectors = std::min<int64_t>(c->nvec, std::min<int64_t>(c->M.nstate, c->n));
  info->h_nnz = c->h_valid ? c->nnz : 0;
  return VHCI_OK;
}

vhci_status vhci_get_stats(const vhci_ctx* c, vhci_stats* s) {
  if (!c || !s) return VHCI_E_INPUT;
  *s = c->stats;
  s->kernel_launches = launch_count();
  return VHCI_OK;
}

vhci_status vhci_reset_stats(vhci_ctx* c) {
  if (!c) return VHCI_E_INPUT;
  c->stats = vhci_stats{};
  return VHCI_OK;
}

static void dump_fc(const std::vector<ForceConstant>& L, double* v, int32_t* m, int32_t* p) {
  for (size_t i = 0; i < L.size(); ++i) {
    v[i] = L[i].fc;
    for (int k = 0; k < kMaxOrder; ++k) {
      m[i * kMaxOrder + k] = k < L[i].nk ? L[i].modes[k] : -1;
      p[i * kMaxOrder + k] = k < L[i].nk ? L[i].powers[k] : 0;
    }
  }
}

vhci_status vhci_get_fc_list(const vhci_ctx* c, double* v, int32_t* m, int32_t* p) {
  if (!c || !v || !m || !p) return VHCI_E_INPUT;
  dump_fc(c->M.fcs, v, m, p);
  return VHCI_OK;
}

vhci_status vhci_get_hb_list(const vhci_ctx* c, double* v, int32_t* m, int32_t* p) {
  if (!c || !v || !m || !p) return VHCI_E_INPUT;
  dump_fc(c->M.hb, v, m, p);
  return VHCI_OK;
}

vhci_status vhci_get_freqs(const vhci_ctx* c, double* f) {
  if (!c || !f) return VHCI_E_INPUT;
  std::copy(c->M.freq.begin(), c->M.freq.end(), f);
  return VHCI_OK;
}

vhci_status vhci_set_basis(vhci_ctx* c, const uint8_t* quanta, int64_t n) {
  if (!c || !quanta || n <= 0) return VHCI_E_INPUT;
  int maxq = 0;
  for (int64_t i = 0; i < n * c->M.nm; ++i) maxq = std::max<int>(maxq, quanta[i]);
  if (maxq > c->L.qmax) {
    c->n = 0;
    VTRY(promote_layout(c));
  }
  DBuf<uint8_t> q;
  VCK(q.reserve(n * c->M.nm, c->st));
  VCK(h2d(c, q.p, quanta, n * c->M.nm));
  VCK(c->keys.reserve((size_t)n * c->L.W, c->st));
  pack_keys(q.p, n, c->M.nm, c->L, c->keys.p, c->st);
  q.release(c->st);
  c->n = n;
  c->hmask = 0;
  VTRY(ensure_hash(c, n));
  int fl = 0;
  VTRY(read_flags(c, &fl));
  c->h_valid = false;
  c->h_prefix = 0;
  c->npanel = 0;
  c->nvec = 0;
  c->x_rows = 0;
  c->E.clear();
  if (fl & kFlagDuplicate) return fail(c, VHCI_E_INPUT, "duplicate states in the basis");
  return VHCI_OK;
}

vhci_status vhci_get_basis(const vhci_ctx* c0, uint8_t* quanta, int64_t cap, int64_t* n) {
  vhci_ctx* c = const_cast<vhci_ctx*>(c0);
  if (!c || !n) return VHCI_E_INPUT;
  *n = c->n;
  if (!quanta) return VHCI_OK;
  if (cap < c->n) return fail(c, VHCI_E_INPUT, "basis buffer too small");
  DBuf<uint8_t> q;
  VCK(q.reserve(std::max<int64_t>(c->n * c->M.nm, 1), c->st));
  unpack_keys(c->keys.p, c->n, c->M.nm, c->L, q.p, c->st);
  VCK(d2h(c, quanta, q.p, c->n * c->M.nm));
  q.release(c->st);
  VCK(cudaStreamSynchronize(c->st));
  return VHCI_OK;
}

vhci_status vhci_set_vectors(vhci_ctx* c, const double* C, const double* E, int k) {
  if (!c || !C || !E || k <= 0) return VHCI_E_INPUT;
  const int64_t n = c->n;
  std::vector<double> h((size_t)n * k);
  for (int64_t i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) h[(size_t)i * k + j] = C[(size_t)j * n + i];
  VCK(c->X.reserve((size_t)n * k, c->st));
  VCK(h2d(c, c->X.p, h.data(), h.size() * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  c->ldx = k;
  c->nvec = k;
  c->x_rows = n;
  c->E.assign(E, E + k);
  return VHCI_OK;
}

vhci_status vhci_get_vectors(const vhci_ctx* c0, double* C, double* E, int k) {
  vhci_ctx* c = const_cast<vhci_ctx*>(c0);
  if (!c) return VHCI_E_INPUT;
  if (k > c->nvec || c->x_rows != c->n) return fail(c, VHCI_E_STATE, "fewer vectors held than requested");
  const int64_t n = c->n;
  if (C) {
    std::vector<double> h((size_t)n * c->ldx);
    VCK(d2h(c, h.data(), c->X.p, h.size() * sizeof(double)));
    VCK(cudaStreamSynchronize(c->st));
    for (int64_t i = 0; i < n; ++i)
      for (int j = 0; j < k; ++j) C[(size_t)j * n + i] = h[(size_t)i * c->ldx + j];
  }
  if (E)
    for (int j = 0; j < k; ++j) E[j] = c->E[j];
  return VHCI_OK;
}

vhci_status vhci_get_energies(const vhci_ctx* c, double* E, int k, int* n) {
  if (!c || !n) return VHCI_E_INPUT;
  const int held = (int)std::min<int64_t>((int64_t)c->E.size(), std::min<int64_t>(c->M.nstate, c->n));
  *n = held;
  if (E)
    for (int j = 0; j < std::min(k, held); ++j) E[j] = c->E[j];
  return VHCI_OK;
}

vhci_status vhci_select(vhci_ctx* c, double eps, int append, int64_t* n_new) {
  if (!c) return VHCI_E_INPUT;
  VCK(cudaEventRecord(c->ev_a, c->st));
  VTRY(generate_new_set(c, eps));
  if (append && c->nsel > 0) {
    VTRY(append_keys(c, c->sel.p, c->nsel));
    // vectors keep their old rows; new rows are zero-extended by the next eigensolve
  }
  VCK(cudaEventRecord(c->ev_b, c->st));
  VCK(cudaEventSynchronize(c->ev_b));
  c->stats.ms_select += event_ms(c);
  int fl = 0;
  VTRY(read_flags(c, &fl));
  if (fl & kFlagTableFull) return fail(c, VHCI_E_TABLE_FULL, "basis hash full");
  if (n_new) *n_new = c->nsel;
  return VHCI_OK;
}

vhci_status vhci_get_selected(const vhci_ctx* c0, uint8_t* quanta, int64_t cap, int64_t* n) {
  vhci_ctx* c = const_cast<vhci_ctx*>(c0);
  if (!c || !n) return VHCI_E_INPUT;
  *n = c->nsel;
  if (!quanta || c->nsel == 0) return VHCI_OK;
  if (cap < c->nsel) return fail(c, VHCI_E_INPUT, "buffer too small");
  DBuf<uint8_t> q;
  VCK(q.reserve(c->nsel * c->M.nm, c->st));
  unpack_keys(c->sel.p, c->nsel, c->M.nm, c->L, q.p, c->st);
  VCK(d2h(c, quanta, q.p, c->nsel * c->M.nm));
  q.release(c->st);
  VCK(cudaStreamSynchronize(c->st));
  return VHCI_OK;
}

vhci_status vhci_build_h(vhci_ctx* c, int64_t* nnz) {
  if (!c) return VHCI_E_INPUT;
  VTRY(build_h(c));
  if (nnz) *nnz = c->nnz + c->n;
  return VHCI_OK;
}

vhci_status vhci_set_comm(vhci_ctx* c, const vhci_comm* comm) {
  if (!c) return VHCI_E_INPUT;
  if (!comm || comm->nranks <= 1) {
    c->comm = vhci_comm{};
  } else {
    if (comm->rank < 0 || comm->rank >= comm->nranks || !comm->allreduce_sum || !comm->allgather)
      return fail(c, VHCI_E_INPUT, "vhci_set_comm: bad rank or missing collective");
    c->comm = *comm;
  }
  c->h_valid = false;  // the held matrix's rows follow the sharding
  c->h_prefix = 0;
  return VHCI_OK;
}

vhci_status vhci_get_h_csr(const vhci_ctx* c0, int64_t* rowptr, int32_t* col, double* val) {
  vhci_ctx* c = const_cast<vhci_ctx*>(c0);
  if (!c || !rowptr || !col || !val) return VHCI_E_INPUT;
  if (!c->h_valid) return fail(c, VHCI_E_STATE, "Hamiltonian not built");
  if (c->h_rows) return fail(c, VHCI_E_STATE, "the Hamiltonian is sharded over the ranks");
  const int64_t n = c->n;
  std::vector<int64_t> rp(n + 1);
  std::vector<int32_t> cl(c->nnz);
  std::vector<double> vl(c->nnz), dg(n);
  VCK(d2h(c, rp.data(), c->rowptr.p, (n + 1) * sizeof(int64_t)));
  if (c->nnz) {
    VCK(d2h(c, cl.data(), c->col.p, c->nnz * sizeof(int32_t)));
    if (c->o.precision == 1) {
      std::vector<float> vf(c->nnz);
      VCK(d2h(c, vf.data(), c->valf.p, c->nnz * sizeof(float)));
      VCK(cudaStreamSynchronize(c->st));
      for (int64_t e = 0; e < c->nnz; ++e) vl[e] = vf[e];
    } else {
      VCK(d2h(c, vl.data(), c->val.p, c->nnz * sizeof(double)));
    }
  }
  VCK(d2h(c, dg.data(), c->diag.p, n * sizeof(double)));
  VCK(cudaStreamSynchronize(c->st));
  int64_t pos = 0;
  std::vector<std::pair<int32_t, double>> row;
  for (int64_t i = 0; i < n; ++i) {
    rowptr[i] = pos;
    row.clear();
    for (int64_t e = rp[i]; e < rp[i + 1]; ++e) row.push_back({cl[e], vl[e]});
    row.push_back({(int32_t)i, dg[i]});
    std::sort(row.begin(), row.end(),
              [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
                return a.first < b.first;
              });
    for (auto& e : row) { col[pos] = e.first; val[pos] = e.second; ++pos; }
  }
  rowptr[n] = pos;
  return VHCI_OK;
}

vhci_status vhci_structural_nnz(vhci_ctx* c, int64_t* nnz) {
  if (!c || !nnz) return VHCI_E_INPUT;
  return structural_count(c, nnz);
}

}  // extern "C"
