// CPU ORACLE — test infrastructure only.  Nothing in the shipped library links or calls this file;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as the checker.
//
// A plain C++17 + OpenMP restatement of the reference VHCI algorithm (berkelbach-group/VHCI),
// written from the published behaviour of its source.  Each function cites the reference file:line
// it restates.  Two forms of the quadratic loops are kept:
//   * "pair" forms follow the reference's O(N^2) pair loops literally (QDiffVec + gates +
//     ScreenState + AnharmPot; src/Ham.cpp:228-326, src/PT2.cpp:66-149), used on small cases and as
//     the timed CPU baseline;
//   * "conn" forms enumerate, per state and force constant, exactly the quanta changes that
//     ScreenState admits, and sum the same terms in the same order, so their results are
//     bit-identical to the pair forms at a cost linear in N.  Tests check the equality.
// Eigen-steps are not here: the Python driver (oracle/oracle.py) uses LAPACK/ARPACK through scipy.
//
// Parity pinning: the Python driver's end-to-end results are compared with outputs of the
// shipped reference binary (tests/golden/), see tests/test_oracle_golden.py.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct FC {
  double fc = 0.0;
  std::vector<int> fcpow;   // mode list, one entry per power (reference FConst::fcpow)
  std::vector<int> modes;   // distinct modes in first-appearance order (ShortModes)
  std::vector<int> powers;  // power of each distinct mode (ModePowers)
};

using State = std::vector<int>;

struct StateHash {
  size_t operator()(const State& s) const {
    uint64_t h = 1469598103934665603ull;
    for (int q : s) { h ^= (uint64_t)(q + 0x9e37); h *= 1099511628211ull; }
    return (size_t)h;
  }
};
using StateSet = std::unordered_set<State, StateHash>;

struct Ctx {
  int nm = 0, ntot = 0, neig = 0, perturb = 0, nfc_in = 0;
  double eps1 = 0.0, eps2 = 0.0;
  std::vector<double> freq;
  std::vector<int> cap;
  std::vector<FC> anharm, hb, cubic, quartic, quintic, sextic;
  std::vector<State> basis;
  int fcmax = 0;
  std::string err;
};

// src/Core_functions.cpp:73-83
double fact(int n) {
  double v = 1;
  while (n > 0) { v *= n; n -= 1; }
  return v;
}

// src/Input_Reader.cpp:249-271 (ShortModes/ModePowers grouping)
void group_modes(FC& f) {
  f.modes.clear(); f.powers.clear();
  for (size_t i = 0; i < f.fcpow.size(); ++i) {
    bool found = false;
    for (size_t j = 0; j < f.modes.size(); ++j)
      if (f.fcpow[i] == f.modes[j]) { f.powers[j] += 1; found = true; }
    if (!found) { f.modes.push_back(f.fcpow[i]); f.powers.push_back(1); }
  }
}

// src/Input_Reader.cpp:494-515 (ScaleFC): fc *= 1/sqrt(2^order) / prod_k p_k!
void scale_fc(std::vector<FC>& fcs) {
  for (auto& f : fcs) {
    double s = (double)f.fcpow.size();
    s = std::pow(2, s);
    s = 1 / std::sqrt(s);
    for (int p : f.powers) s /= fact(p);
    f.fc *= s;
  }
}

// src/Input_Reader.cpp:295-364: all product states with sum of quanta <= Ntot, per-mode quanta
// <= min(cap, Ntot); order: mode 0 innermost-first, each new mode's quanta in the outer loop.
void initial_basis(Ctx& c) {
  c.basis.clear();
  int nexc = std::min(c.cap[0] + 1, c.ntot + 1);
  for (int i = 0; i < nexc; ++i) c.basis.push_back(State{i});
  for (int m = 1; m < c.nm; ++m) {
    std::vector<State> nb;
    nexc = std::min(c.cap[m] + 1, c.ntot + 1);
    for (int j = 0; j < nexc; ++j)
      for (const State& s : c.basis) {
        State t = s; t.push_back(j);
        int tot = 0; for (int q : t) tot += q;
        if (tot <= c.ntot) nb.push_back(t);
      }
    c.basis.swap(nb);
  }
}

// src/Input_Reader.cpp:366-460: heat-bath list = scaled FCs + aggregated single and double terms.
void build_hb(Ctx& c) {
  c.hb = c.anharm;
  for (int m = 0; m < c.nm; ++m) {  // singles: 3 V_mmm + 2 V_m(nn)
    FC t; t.fcpow = {m}; t.modes = {m}; t.powers = {1}; t.fc = 0.;
    for (const FC& f : c.cubic) {
      if (f.modes.size() == 1 && f.modes[0] == m) t.fc += 3 * f.fc;
      if (f.modes.size() == 2)
        for (int i = 0; i < 2; ++i)
          if (f.modes[i] == m && f.powers[i] == 1) { t.fc += 2 * f.fc; break; }
    }
    if (std::fabs(t.fc) > 1e-8) c.hb.push_back(t);
  }
  for (int m = 0; m < c.nm; ++m) {  // doubles m=n: 4 V_mmmm + 2 V_mmnn
    FC t; t.fcpow = {m, m}; t.modes = {m}; t.powers = {2}; t.fc = 0.;
    for (const FC& f : c.quartic) {
      if (f.modes.size() == 1 && f.modes[0] == m) t.fc += 4 * f.fc;
      if (f.modes.size() == 2)
        for (int i = 0; i < 2; ++i)
          if (f.modes[i] == m && f.powers[i] == 2) { t.fc += 2 * f.fc; break; }
    }
    if (std::fabs(t.fc) > 1e-8) c.hb.push_back(t);
  }
  for (int m = 0; m + 1 < c.nm; ++m)  // doubles m!=n: 3 V_mnnn / V_mmmn + 2 V_mnll
    for (int n = m + 1; n < c.nm; ++n) {
      FC t; t.fcpow = {m, n}; t.modes = {m, n}; t.powers = {1, 1}; t.fc = 0.;
      for (const FC& f : c.quartic) {
        bool pow3 = std::find(f.powers.begin(), f.powers.end(), 3) != f.powers.end();
        auto im = std::find(f.modes.begin(), f.modes.end(), m);
        auto in = std::find(f.modes.begin(), f.modes.end(), n);
        bool fm = im != f.modes.end(), fn = in != f.modes.end();
        if (f.modes.size() == 2 && pow3 && fm && fn) t.fc += 3 * f.fc;
        if (f.modes.size() == 3 && fm && fn && f.powers[im - f.modes.begin()] == 1 &&
            f.powers[in - f.modes.begin()] == 1)
          t.fc += 2 * f.fc;
      }
      if (std::fabs(t.fc) > 1e-8) c.hb.push_back(t);
    }
  // src/HB.cpp:17-22: sort by |fc| descending (ties only reorder equal thresholds)
  std::stable_sort(c.hb.begin(), c.hb.end(),
                   [](const FC& a, const FC& b) { return std::fabs(a.fc) > std::fabs(b.fc); });
}

// src/Input_Reader.cpp:170-291 positional parse.  Returns false with c.err set on failure.
bool parse(Ctx& c, const char* path) {
  std::ifstream in(path);
  if (!in.good()) { c.err = "Could not open input file."; return false; }
  std::string dummy;
  std::getline(in, dummy);
  in >> dummy >> c.eps1 >> dummy >> c.neig >> dummy >> c.perturb >> dummy >> c.eps2;
  if (c.perturb != 0 && c.perturb != 1) { c.err = "perturb must be either 0 or 1"; return false; }
  if (c.perturb == 0) c.eps2 = 0;
  in >> dummy >> c.ntot >> dummy >> c.nm;
  for (int i = 0; i < c.nm; ++i) {
    int id; double f; int q;
    in >> id >> f >> q;
    if (id != i) { c.err = "Expected mode " + std::to_string(i); return false; }
    c.freq.push_back(f); c.cap.push_back(q);
  }
  in >> dummy >> c.nfc_in;
  for (int i = 0; i < c.nfc_in; ++i) {
    FC f; int p = 0; in >> p;
    for (int j = 0; j < p; ++j) { int m; in >> m; f.fcpow.push_back(m); }
    in >> f.fc;
    c.anharm.push_back(f);
  }
  if (!in) { c.err = "truncated input"; return false; }
  for (auto& f : c.anharm) group_modes(f);
  scale_fc(c.anharm);
  for (const FC& f : c.anharm) {
    switch (f.fcpow.size()) {
      case 3: c.cubic.push_back(f); break;
      case 4: c.quartic.push_back(f); break;
      case 5: c.quintic.push_back(f); break;
      case 6: c.sextic.push_back(f); break;
      default: c.err = "Force constants are only supported up to 6th order!"; return false;
    }
  }
  c.fcmax = 0;  // src/Ham.cpp:231-236
  for (const FC& f : c.anharm) c.fcmax = std::max<int>(c.fcmax, (int)f.fcpow.size());
  initial_basis(c);
  build_hb(c);
  return true;
}

// src/Ham.cpp:38-104 AnharmPot: fc * prod_k <m_k| (a + a^dag)^{p_k} |n_k>, by path expansion
// (creation branch before annihilation branch at each step).
double anharm_pot(const State& n, const State& m, const FC& f) {
  double v = f.fc;
  std::vector<double> csum(f.modes.size(), 0.0);
  for (size_t i = 0; i < f.modes.size(); ++i) {
    std::vector<int> st{n[f.modes[i]]};
    std::vector<double> co{1.0};
    for (int j = 0; j < f.powers[i]; ++j) {
      std::vector<int> s2; std::vector<double> c2;
      for (size_t k = 0; k < st.size(); ++k) {
        int q = st[k]; double cc = co[k];
        cc *= std::sqrt(q + 1); q += 1;  // CreationLO
        s2.push_back(q); c2.push_back(cc);
        q = st[k]; cc = co[k];
        cc *= std::sqrt(q); q -= 1;       // AnnihilationLO
        if (q < 0) { q = -1; cc = 0; }
        if (q >= 0) { s2.push_back(q); c2.push_back(cc); }
      }
      st.swap(s2); co.swap(c2);
    }
    for (size_t j = 0; j < st.size(); ++j)
      if (st[j] == m[f.modes[i]]) csum[i] += co[j];
  }
  for (double cs : csum) v *= cs;
  return v;
}

// src/Ham.cpp:381-399
void qdiff_vec(const State& a, const State& b, int& qtot, int& mchange, std::vector<int>& d) {
  qtot = 0; mchange = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    int q = a[i] - b[i];
    d[i] = std::abs(q);
    qtot += std::abs(q);
    if (q != 0) mchange += 1;
  }
}

// src/Ham.cpp:401-446
bool screen_state(int qdiff, int mchange, const std::vector<int>& d, const FC& f) {
  if (qdiff > (int)f.fcpow.size() || mchange > (int)f.modes.size() ||
      qdiff % 2 != (int)f.fcpow.size() % 2)
    return false;
  for (size_t i = 0; i < f.modes.size(); ++i)
    if (d[f.modes[i]] > f.powers[i] || d[f.modes[i]] % 2 != f.powers[i] % 2) return false;
  for (int i = 0; i < (int)d.size(); ++i) {
    bool in_fc = false;
    for (int m : f.modes) if (m == i) { in_fc = true; break; }
    if (!in_fc && d[i] != 0) return false;
  }
  return true;
}

double harmonic(const Ctx& c, const State& s) {  // src/Ham.cpp:211-220
  double e = 0.;
  for (int j = 0; j < c.nm; ++j) { double ej = 0.5; ej += s[j]; ej *= c.freq[j]; e += ej; }
  return e;
}

// Sum of admitted terms for one pair, as in src/Ham.cpp:247-322: even quanta change sums
// quartic then sextic terms under the gate qdiff<=fcmax, mchange<=fcmax; odd sums cubic then
// quintic under qdiff<=fcmax-1, mchange<=fcmax-1.  `ket` is the state the operators act on.
// Returns false when the pair fails the gate (no structural entry).
bool pair_value(const Ctx& c, const State& ket, const State& bra, std::vector<int>& d, double& v) {
  int qd = 0, mc = 0;
  qdiff_vec(ket, bra, qd, mc, d);
  v = 0;
  if (qd <= c.fcmax && mc <= c.fcmax && qd % 2 == 0) {
    for (const FC& f : c.quartic) if (screen_state(qd, mc, d, f)) v += anharm_pot(ket, bra, f);
    for (const FC& f : c.sextic) if (screen_state(qd, mc, d, f)) v += anharm_pot(ket, bra, f);
    return true;
  }
  if (qd <= c.fcmax - 1 && mc <= c.fcmax - 1 && qd % 2 == 1) {
    for (const FC& f : c.cubic) if (screen_state(qd, mc, d, f)) v += anharm_pot(ket, bra, f);
    for (const FC& f : c.quintic) if (screen_state(qd, mc, d, f)) v += anharm_pot(ket, bra, f);
    return true;
  }
  return false;
}

// Enumerate the quanta-change patterns of one FC: every delta_k in {-p_k, -p_k+2, ..., p_k}
// (src/HB.cpp:27-164 and the ScreenState conditions of src/Ham.cpp:401-446).
template <class F>
void for_each_pattern(const FC& f, F&& fn) {
  int nk = (int)f.modes.size();
  int d[6];
  for (int k = 0; k < nk; ++k) d[k] = -f.powers[k];
  while (true) {
    fn(d, nk);
    int k = nk - 1;
    while (k >= 0) {
      d[k] += 2;
      if (d[k] <= f.powers[k]) break;
      d[k] = -f.powers[k];
      --k;
    }
    if (k < 0) break;
  }
}

// True when the reference's pair gate admits a change pattern with the given parity
// (src/Ham.cpp:247,283): for odd patterns the gate is qdiff<=fcmax-1 and mchange<=fcmax-1.
bool gate_ok(const Ctx& c, const int* d, int nk) {
  int qd = 0, mc = 0;
  for (int k = 0; k < nk; ++k) { qd += std::abs(d[k]); if (d[k]) ++mc; }
  if (qd % 2 == 0) return qd <= c.fcmax && mc <= c.fcmax;
  return qd <= c.fcmax - 1 && mc <= c.fcmax - 1;
}

struct Handle {
  Ctx c;
  // results kept for copy-out
  std::vector<State> out_states;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<double> val;
  int64_t structural = 0;
};

std::unordered_map<State, int64_t, StateHash> index_of(const std::vector<State>& b) {
  std::unordered_map<State, int64_t, StateHash> m;
  m.reserve(b.size() * 2);
  for (size_t i = 0; i < b.size(); ++i) m.emplace(b[i], (int64_t)i);
  return m;
}

// src/HB.cpp:204-214: signed entry of max |C_ij| over j < nopt, first occurrence wins.
std::vector<double> cmax_rows(const double* C, int64_t n, int ncols, int nopt) {
  std::vector<double> cm(n);
  for (int64_t i = 0; i < n; ++i) {
    double cij = C[i];
    for (int j = 1; j < nopt && j < ncols; ++j)
      if (std::fabs(C[i + (int64_t)j * n]) > std::fabs(cij)) cij = C[i + (int64_t)j * n];
    cm[i] = cij;
  }
  return cm;
}

// src/HB.cpp:24-174 AddStatesHB for every state n (serial, as the reference's driver loop).
void add_states_hb(const Ctx& c, const std::vector<double>& cmax, double eps, StateSet& init,
                   StateSet& out) {
  for (size_t n = 0; n < c.basis.size(); ++n) {
    double cn = cmax[n];
    for (const FC& f : c.hb) {
      if (!(std::fabs(cn * f.fc) >= eps)) break;
      for_each_pattern(f, [&](const int* d, int nk) {
        bool zero = true;
        for (int k = 0; k < nk; ++k) if (d[k]) zero = false;
        if (zero) return;
        State t = c.basis[n];
        for (int k = 0; k < nk; ++k) {
          t[f.modes[k]] += d[k];
          if (t[f.modes[k]] < 0) return;
        }
        if (init.count(t) == 0) out.insert(t);
      });
    }
  }
}

}  // namespace

extern "C" {

void* orc_load(const char* path, char* err, int errlen) {
  Handle* h = new Handle();
  if (!parse(h->c, path)) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", h->c.err.c_str());
    delete h;
    return nullptr;
  }
  return h;
}

void orc_free(void* p) { delete (Handle*)p; }

// info: [nm, ntot, neig, perturb, n_basis, n_fc, n_hb, fcmax]; dinfo: [eps1, eps2]
void orc_info(void* p, int64_t* info, double* dinfo) {
  Ctx& c = ((Handle*)p)->c;
  info[0] = c.nm; info[1] = c.ntot; info[2] = c.neig; info[3] = c.perturb;
  info[4] = (int64_t)c.basis.size(); info[5] = (int64_t)c.anharm.size();
  info[6] = (int64_t)c.hb.size(); info[7] = c.fcmax;
  dinfo[0] = c.eps1; dinfo[1] = c.eps2;
}

void orc_freqs(void* p, double* f) {
  Ctx& c = ((Handle*)p)->c;
  for (int i = 0; i < c.nm; ++i) f[i] = c.freq[i];
}

// Heat-bath list after sorting: values and mode/power descriptors (6 slots, -1 padded).
void orc_hb_list(void* p, double* fc, int32_t* modes, int32_t* powers) {
  Ctx& c = ((Handle*)p)->c;
  for (size_t i = 0; i < c.hb.size(); ++i) {
    fc[i] = c.hb[i].fc;
    for (int k = 0; k < 6; ++k) {
      bool v = k < (int)c.hb[i].modes.size();
      modes[i * 6 + k] = v ? c.hb[i].modes[k] : -1;
      powers[i * 6 + k] = v ? c.hb[i].powers[k] : 0;
    }
  }
}

// Scaled FC list in input order.
void orc_fc_list(void* p, double* fc, int32_t* modes, int32_t* powers) {
  Ctx& c = ((Handle*)p)->c;
  for (size_t i = 0; i < c.anharm.size(); ++i) {
    fc[i] = c.anharm[i].fc;
    for (int k = 0; k < 6; ++k) {
      bool v = k < (int)c.anharm[i].modes.size();
      modes[i * 6 + k] = v ? c.anharm[i].modes[k] : -1;
      powers[i * 6 + k] = v ? c.anharm[i].powers[k] : 0;
    }
  }
}

int64_t orc_basis_size(void* p) { return (int64_t)((Handle*)p)->c.basis.size(); }

void orc_get_basis(void* p, int32_t* q) {
  Ctx& c = ((Handle*)p)->c;
  for (size_t i = 0; i < c.basis.size(); ++i)
    for (int m = 0; m < c.nm; ++m) q[i * c.nm + m] = c.basis[i][m];
}

void orc_set_basis(void* p, const int32_t* q, int64_t n) {
  Ctx& c = ((Handle*)p)->c;
  c.basis.assign(n, State(c.nm));
  for (int64_t i = 0; i < n; ++i)
    for (int m = 0; m < c.nm; ++m) c.basis[i][m] = q[i * c.nm + m];
}

void orc_append_basis(void* p, const int32_t* q, int64_t n) {
  Ctx& c = ((Handle*)p)->c;
  for (int64_t i = 0; i < n; ++i) {
    State s(c.nm);
    for (int m = 0; m < c.nm; ++m) s[m] = q[i * c.nm + m];
    c.basis.push_back(s);
  }
}

// Heat-bath selection over the current basis with caller-supplied vectors C (n x ncols,
// column-major) and nopt columns.  New states are kept in the handle, sorted lexicographically
// (mode 0 most significant); returns their count.
int64_t orc_select(void* p, const double* C, int ncols, int nopt, double eps) {
  Handle* h = (Handle*)p;
  Ctx& c = h->c;
  auto cm = cmax_rows(C, (int64_t)c.basis.size(), ncols, nopt);
  StateSet init(c.basis.begin(), c.basis.end()), out;
  add_states_hb(c, cm, eps, init, out);
  h->out_states.assign(out.begin(), out.end());
  std::sort(h->out_states.begin(), h->out_states.end());
  return (int64_t)h->out_states.size();
}

void orc_get_selected(void* p, int32_t* q) {
  Handle* h = (Handle*)p;
  int nm = h->c.nm;
  for (size_t i = 0; i < h->out_states.size(); ++i)
    for (int m = 0; m < nm; ++m) q[i * nm + m] = h->out_states[i][m];
}

// Dense H over the current basis (src/Ham.cpp:107-200: ZerothHam + AnharmHam), row-major n x n.
void orc_dense_h(void* p, double* H) {
  Ctx& c = ((Handle*)p)->c;
  int64_t n = (int64_t)c.basis.size();
  std::memset(H, 0, sizeof(double) * n * n);
  for (int64_t i = 0; i < n; ++i) H[i * n + i] += harmonic(c, c.basis[i]);
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t i = 0; i < n; ++i) {
    std::vector<int> d(c.nm);
    for (int64_t j = i; j < n; ++j) {
      double v;
      if (pair_value(c, c.basis[i], c.basis[j], d, v)) {
        H[i * n + j] += v;
        if (i != j) H[j * n + i] += v;
      }
    }
  }
}

// Sparse H, literal pair loop (src/Ham.cpp:203-344).  Stores the full symmetric matrix as CSR with
// entries for every gated pair (structural zeros included, as Eigen keeps them) and returns nnz.
// Diagonal = fl(E_harm/2 + V_ii/2) * 2 as in the triplet assembly; off-diagonal = V_ij with the
// lower-index state as the ket.
int64_t orc_build_h_pairs(void* p) {
  Handle* h = (Handle*)p;
  Ctx& c = h->c;
  int64_t n = (int64_t)c.basis.size();
  std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
  std::vector<double> diag(n);
  for (int64_t i = 0; i < n; ++i) diag[i] = harmonic(c, c.basis[i]) / 2.;
#pragma omp parallel
  {
    std::vector<int> d(c.nm);
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
      for (int64_t j = i; j < n; ++j) {
        double v;
        if (!pair_value(c, c.basis[i], c.basis[j], d, v)) continue;
        if (i == j) diag[i] = (diag[i] + v / 2.) * 2.;
        else rows[i].push_back({(int32_t)j, v});
      }
    }
  }
  // mirror the upper triangle (H + H^T of src/Ham.cpp:336-338)
  std::vector<std::vector<std::pair<int32_t, double>>> full(n);
  for (int64_t i = 0; i < n; ++i) {
    for (auto& e : rows[i]) { full[i].push_back(e); full[e.first].push_back({(int32_t)i, e.second}); }
  }
  h->rowptr.assign(n + 1, 0);
  h->col.clear(); h->val.clear();
  for (int64_t i = 0; i < n; ++i) {
    full[i].push_back({(int32_t)i, diag[i]});
    std::sort(full[i].begin(), full[i].end(),
              [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
                return a.first < b.first;
              });
    for (auto& e : full[i]) { h->col.push_back(e.first); h->val.push_back(e.second); }
    h->rowptr[i + 1] = (int64_t)h->col.size();
  }
  h->structural = (int64_t)h->col.size();
  return h->structural;
}

// Sparse H by connection enumeration: same entries (only pairs connected by >= 1 admitted FC,
// plus the diagonal), same per-pair summation order (quartic, sextic | cubic, quintic lists in
// input order) and the same ket convention (lower basis index), so values equal the pair form's.
int64_t orc_build_h_conn(void* p) {
  Handle* h = (Handle*)p;
  Ctx& c = h->c;
  int64_t n = (int64_t)c.basis.size();
  auto idx = index_of(c.basis);
  std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
  const std::vector<FC>* lists[4] = {&c.quartic, &c.sextic, &c.cubic, &c.quintic};
#pragma omp parallel
  {
    std::vector<int> d(c.nm);
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
      std::vector<int32_t> hits;
      // targets j connected to i by at least one admitted FC
      std::unordered_set<int32_t> seen;
      for (auto* L : lists)
        for (const FC& f : *L)
          for_each_pattern(f, [&](const int* dd, int nk) {
            if (!gate_ok(c, dd, nk)) return;
            State t = c.basis[i];
            for (int k = 0; k < nk; ++k) {
              t[f.modes[k]] += dd[k];
              if (t[f.modes[k]] < 0) return;
            }
            auto it = idx.find(t);
            if (it == idx.end()) return;
            if (seen.insert((int32_t)it->second).second) hits.push_back((int32_t)it->second);
          });
      std::sort(hits.begin(), hits.end());
      for (int32_t j : hits) {
        double v;
        const State& ket = (j < i) ? c.basis[j] : c.basis[i];
        const State& bra = (j < i) ? c.basis[i] : c.basis[j];
        pair_value(c, ket, bra, d, v);
        if (j == i) v = (harmonic(c, c.basis[i]) / 2. + v / 2.) * 2.;
        rows[i].push_back({j, v});
      }
      if (!seen.count((int32_t)i)) {  // diagonal with no even FC term
        rows[i].push_back({(int32_t)i, (harmonic(c, c.basis[i]) / 2.) * 2.});
        std::sort(rows[i].begin(), rows[i].end(),
                  [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
                    return a.first < b.first;
                  });
      }
    }
  }
  h->rowptr.assign(n + 1, 0);
  h->col.clear(); h->val.clear();
  for (int64_t i = 0; i < n; ++i) {
    for (auto& e : rows[i]) { h->col.push_back(e.first); h->val.push_back(e.second); }
    h->rowptr[i + 1] = (int64_t)h->col.size();
  }
  return (int64_t)h->col.size();
}

void orc_get_csr(void* p, int64_t* rowptr, int32_t* col, double* val) {
  Handle* h = (Handle*)p;
  std::memcpy(rowptr, h->rowptr.data(), sizeof(int64_t) * h->rowptr.size());
  std::memcpy(col, h->col.data(), sizeof(int32_t) * h->col.size());
  std::memcpy(val, h->val.data(), sizeof(double) * h->val.size());
}

// Epstein-Nesbet PT2 (src/PT2.cpp:16-154) with caller-supplied variational vectors C (n x ncols,
// column-major) and energies E.  Perturbers P come from AddStatesHB with eps2 (src/PT2.cpp:29-50).
// mode 0: literal (a, i) pair loop; mode 1: connection enumeration with i summed in ascending
// order (bit-identical).  dE[n] for n < nopt; returns |P|.  The perturber set is kept (sorted).
int64_t orc_pt2(void* p, const double* C, int ncols, const double* E, int nopt, double eps2,
                int mode, double* dE) {
  Handle* h = (Handle*)p;
  Ctx& c = h->c;
  int64_t n = (int64_t)c.basis.size();
  auto cm = cmax_rows(C, n, ncols, nopt);
  StateSet init(c.basis.begin(), c.basis.end()), pset;
  add_states_hb(c, cm, eps2, init, pset);
  std::vector<State> P(pset.begin(), pset.end());
  std::sort(P.begin(), P.end());
  h->out_states = P;
  int64_t np = (int64_t)P.size();
  std::vector<double> acc(nopt, 0.0);
  auto idx = index_of(c.basis);
  const std::vector<FC>* lists[4] = {&c.quartic, &c.sextic, &c.cubic, &c.quintic};
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  std::vector<std::vector<double>> part(nthreads, std::vector<double>(nopt, 0.0));
  // deterministic: per-thread partials over contiguous chunks of a, reduced in thread order
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    std::vector<int> d(c.nm);
    std::vector<double> sum(nopt);
#pragma omp for schedule(static)
    for (int64_t a = 0; a < np; ++a) {
      std::fill(sum.begin(), sum.end(), 0.0);
      const State& sa = P[a];
      if (mode == 0) {
        for (int64_t i = 0; i < n; ++i) {
          double hai;
          if (!pair_value(c, sa, c.basis[i], d, hai)) continue;
          for (int k = 0; k < nopt; ++k) sum[k] += hai * C[i + (int64_t)k * n];
        }
      } else {
        std::vector<int64_t> hits;
        std::unordered_set<int64_t> seen;
        for (auto* L : lists)
          for (const FC& f : *L)
            for_each_pattern(f, [&](const int* dd, int nk) {
              if (!gate_ok(c, dd, nk)) return;
              State t = sa;
              for (int k = 0; k < nk; ++k) {
                t[f.modes[k]] += dd[k];
                if (t[f.modes[k]] < 0) return;
              }
              auto it = idx.find(t);
              if (it == idx.end()) return;
              if (seen.insert(it->second).second) hits.push_back(it->second);
            });
        std::sort(hits.begin(), hits.end());
        for (int64_t i : hits) {
          double hai;
          pair_value(c, sa, c.basis[i], d, hai);
          for (int k = 0; k < nopt; ++k) sum[k] += hai * C[i + (int64_t)k * n];
        }
      }
      // E_a = harmonic + even-order diagonal terms (src/PT2.cpp:119-144)
      double ea = harmonic(c, sa);
      std::vector<int> z(c.nm, 0);
      for (const FC& f : c.quartic) if (screen_state(0, 0, z, f)) ea += anharm_pot(sa, sa, f);
      for (const FC& f : c.sextic) if (screen_state(0, 0, z, f)) ea += anharm_pot(sa, sa, f);
      for (int k = 0; k < nopt; ++k) part[tid][k] += std::pow(sum[k], 2) / (E[k] - ea);
    }
  }
  for (int t = 0; t < nthreads; ++t)
    for (int k = 0; k < nopt; ++k) acc[k] += part[t][k];
  for (int k = 0; k < nopt; ++k) dE[k] = acc[k];
  return np;
}

// Timed sample of the reference's pair loop (src/Ham.cpp:237-323, the same body as
// src/PT2.cpp:70-118): rows i = r0, r0+stride, ... < r1, each against every j >= i, in parallel
// over rows.  Returns the number of (i, j) pairs evaluated; *checksum receives the sum of values.
int64_t orc_pair_rows(void* p, int64_t r0, int64_t r1, int64_t stride, double* checksum) {
  Ctx& c = ((Handle*)p)->c;
  const int64_t n = (int64_t)c.basis.size();
  int64_t pairs = 0;
  double sum = 0.0;
#pragma omp parallel reduction(+ : pairs, sum)
  {
    std::vector<int> d(c.nm);
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = r0; i < r1; i += stride) {
      for (int64_t j = i; j < n; ++j) {
        double v;
        if (pair_value(c, c.basis[i], c.basis[j], d, v)) sum += v;
      }
      pairs += n - i;
    }
  }
  if (checksum) *checksum = sum;
  return pairs;
}

// Ladder factor <n+delta| (a + a^dag)^p |n> by the reference's path expansion (src/Ham.cpp:38-104).
double orc_ladder(int p, int n, int delta) {
  FC f; f.fc = 1.0; f.fcpow.assign(p, 0); f.modes = {0}; f.powers = {p};
  State a{n}, b{n + delta};
  return anharm_pot(a, b, f);
}

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
