// Host-side problem model.  Semantics follow the reference's Input_Reader.cpp, HB.cpp and Ham.cpp
// (file:line cited per function); the data layout is this library's own.
#include "model.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <functional>
#include <map>

namespace vhci {

namespace {

double factorial(int n) {  // Core_functions.cpp:73-83 (descending product)
  double v = 1;
  for (; n > 0; --n) v *= n;
  return v;
}

// Distinct modes in first-appearance order with their multiplicity (Input_Reader.cpp:249-271).
void group_modes(const int* idx, int order, ForceConstant& f) {
  f.order = order;
  f.nk = 0;
  for (int i = 0; i < order; ++i) {
    int k = 0;
    while (k < f.nk && f.modes[k] != idx[i]) ++k;
    if (k == f.nk) { f.modes[f.nk] = idx[i]; f.powers[f.nk] = 0; ++f.nk; }
    f.powers[k] += 1;
  }
}

// Mixed-radix walk over the patterns of one (modes, powers) set, last mode fastest.
template <class Fn>
void for_each_pattern(int nk, const int* powers, Fn&& fn) {
  int d[kMaxOrder];
  for (int k = 0; k < nk; ++k) d[k] = -powers[k];
  for (;;) {
    fn(d);
    int k = nk - 1;
    for (; k >= 0; --k) {
      d[k] += 2;
      if (d[k] <= powers[k]) break;
      d[k] = -powers[k];
    }
    if (k < 0) return;
  }
}

}  // namespace

bool parse_input_file(const char* path, Model& m, std::string& err) {
  std::ifstream in(path);
  if (!in.good()) { err = "Error: Could not open input file."; return false; }
  std::string tok;
  std::getline(in, tok);  // comment line
  int perturb = 0;
  in >> tok >> m.eps1 >> tok >> m.nstate >> tok >> perturb >> tok >> m.eps2;
  if (!in) { err = "Error: malformed input header."; return false; }
  if (perturb != 0 && perturb != 1) { err = "Error: perturb must be either 0 or 1 "; return false; }
  m.pt2 = perturb;
  if (m.pt2 == 0) m.eps2 = 0;  // Input_Reader.cpp:199-201
  in >> tok >> m.ntot >> tok >> m.nm;
  if (!in || m.nm <= 0) { err = "Error: malformed mode block."; return false; }
  for (int i = 0; i < m.nm; ++i) {
    int id = -1, q = 0;
    double f = 0;
    in >> id >> f >> q;
    if (!in) { err = "Error: malformed mode block."; return false; }
    if (id != i) {
      err = "Error: Expected mode " + std::to_string(i) + " but read data for mode " +
            std::to_string(id);
      return false;
    }
    m.freq.push_back(f);
    m.cap.push_back(q);
  }
  in >> tok >> m.nfc_in;
  if (!in || m.nfc_in < 0) { err = "Error: malformed force-constant block."; return false; }
  for (int i = 0; i < m.nfc_in; ++i) {
    int order = 0;
    in >> order;
    if (!in) { err = "Error: truncated force-constant block."; return false; }
    if (order < 3 || order > kMaxOrder) {
      err = "Error: Force constants are only supported up to 6th order!";
      return false;
    }
    int idx[kMaxOrder];
    for (int j = 0; j < order; ++j) in >> idx[j];
    ForceConstant f;
    in >> f.fc;
    if (!in) { err = "Error: truncated force-constant block."; return false; }
    for (int j = 0; j < order; ++j)
      if (idx[j] < 0 || idx[j] >= m.nm) { err = "Error: force constant names an unknown mode."; return false; }
    group_modes(idx, order, f);
    m.fcs.push_back(f);
  }
  return true;
}

bool model_from_problem(const vhci_problem* p, Model& m, std::string& err) {
  if (!p || p->nmodes <= 0 || !p->freq || !p->cap || p->nfc < 0) { err = "Error: bad problem."; return false; }
  m.nm = p->nmodes;
  m.ntot = p->max_quanta;
  m.nstate = p->nstate;
  m.pt2 = p->pt2 ? 1 : 0;
  m.eps1 = p->eps1;
  m.eps2 = m.pt2 ? p->eps2 : 0.0;
  m.freq.assign(p->freq, p->freq + m.nm);
  m.cap.assign(p->cap, p->cap + m.nm);
  m.nfc_in = p->nfc;
  for (int i = 0; i < p->nfc; ++i) {
    int order = p->fc_order[i];
    if (order < 3 || order > kMaxOrder) {
      err = "Error: Force constants are only supported up to 6th order!";
      return false;
    }
    ForceConstant f;
    f.fc = p->fc_value[i];
    for (int j = 0; j < order; ++j) {
      int md = p->fc_modes[i * kMaxOrder + j];
      if (md < 0 || md >= m.nm) { err = "Error: force constant names an unknown mode."; return false; }
    }
    group_modes(p->fc_modes + i * kMaxOrder, order, f);
    m.fcs.push_back(f);
  }
  return true;
}

// Input_Reader.cpp:295-364: states with sum of quanta <= Ntot and quanta <= min(cap, Ntot) per
// mode.  Mode m is appended with its quanta j in the outer loop over the existing list.
static void make_initial_basis(Model& m, bool restart) {
  const int nm = m.nm;
  std::vector<std::vector<uint8_t>> cur;
  if (restart) {
    cur.push_back(std::vector<uint8_t>(nm, 0));
  } else {
    int nexc = std::min(m.cap[0] + 1, m.ntot + 1);
    for (int i = 0; i < nexc; ++i) cur.push_back(std::vector<uint8_t>{(uint8_t)i});
    for (int md = 1; md < nm; ++md) {
      std::vector<std::vector<uint8_t>> next;
      nexc = std::min(m.cap[md] + 1, m.ntot + 1);
      for (int j = 0; j < nexc; ++j)
        for (const auto& s : cur) {
          int tot = j;
          for (uint8_t q : s) tot += q;
          if (tot <= m.ntot) {
            next.push_back(s);
            next.back().push_back((uint8_t)j);
          }
        }
      cur.swap(next);
    }
  }
  m.n0 = (int64_t)cur.size();
  m.init_basis.resize((size_t)m.n0 * nm);
  for (int64_t i = 0; i < m.n0; ++i)
    std::copy(cur[i].begin(), cur[i].end(), m.init_basis.begin() + i * nm);
}

// Input_Reader.cpp:366-460 aggregated single/double excitation terms appended to the FC list,
// then HB.cpp:17-22 ordering by |fc| descending.
static void make_hb_list(Model& m) {
  m.hb = m.fcs;
  auto push_if = [&](ForceConstant t) {
    if (std::fabs(t.fc) > 1e-8) m.hb.push_back(t);
  };
  for (int md = 0; md < m.nm; ++md) {  // single: 3 V_mmm + 2 V_mnn / V_mmn with p_m = 1
    ForceConstant t;
    t.order = 1; t.nk = 1; t.modes[0] = md; t.powers[0] = 1;
    for (const auto& f : m.fcs) {
      if (f.order != 3) continue;
      if (f.nk == 1 && f.modes[0] == md) t.fc += 3 * f.fc;
      if (f.nk == 2)
        for (int i = 0; i < 2; ++i)
          if (f.modes[i] == md && f.powers[i] == 1) { t.fc += 2 * f.fc; break; }
    }
    push_if(t);
  }
  for (int md = 0; md < m.nm; ++md) {  // double, same mode: 4 V_mmmm + 2 V_mmnn
    ForceConstant t;
    t.order = 2; t.nk = 1; t.modes[0] = md; t.powers[0] = 2;
    for (const auto& f : m.fcs) {
      if (f.order != 4) continue;
      if (f.nk == 1 && f.modes[0] == md) t.fc += 4 * f.fc;
      if (f.nk == 2)
        for (int i = 0; i < 2; ++i)
          if (f.modes[i] == md && f.powers[i] == 2) { t.fc += 2 * f.fc; break; }
    }
    push_if(t);
  }
  for (int a = 0; a + 1 < m.nm; ++a)  // double, two modes: 3 V_mnnn / V_mmmn + 2 V_mnll
    for (int b = a + 1; b < m.nm; ++b) {
      ForceConstant t;
      t.order = 2; t.nk = 2; t.modes[0] = a; t.modes[1] = b; t.powers[0] = 1; t.powers[1] = 1;
      for (const auto& f : m.fcs) {
        if (f.order != 4) continue;
        int ia = -1, ib = -1;
        bool has3 = false;
        for (int k = 0; k < f.nk; ++k) {
          if (f.modes[k] == a) ia = k;
          if (f.modes[k] == b) ib = k;
          if (f.powers[k] == 3) has3 = true;
        }
        if (f.nk == 2 && has3 && ia >= 0 && ib >= 0) t.fc += 3 * f.fc;
        if (f.nk == 3 && ia >= 0 && ib >= 0 && f.powers[ia] == 1 && f.powers[ib] == 1)
          t.fc += 2 * f.fc;
      }
      push_if(t);
    }
  std::stable_sort(m.hb.begin(), m.hb.end(), [](const ForceConstant& x, const ForceConstant& y) {
    return std::fabs(x.fc) > std::fabs(y.fc);
  });
}

bool finalize_model(Model& m, bool restart, std::string& err) {
  // ScaleFC (Input_Reader.cpp:494-515), same operation order: pow(2, order), 1/sqrt, then
  // successive division by the factorial of each mode power.
  for (auto& f : m.fcs) {
    double s = (double)f.order;
    s = std::pow(2, s);
    s = 1 / std::sqrt(s);
    for (int k = 0; k < f.nk; ++k) s /= factorial(f.powers[k]);
    f.fc *= s;
  }
  m.fcmax = 0;
  for (const auto& f : m.fcs) m.fcmax = std::max(m.fcmax, f.order);
  if (m.nstate < 1) { err = "Error: Nstate must be at least 1."; return false; }
  make_initial_basis(m, restart);
  make_hb_list(m);
  return true;
}

// Orders t.groups by lowered-mode key (stable: first-seen order within a segment), records the
// segments, and lays out the terms contiguously per group (per_group: terms of each group in the
// original order, or null for groups without terms).
static void index_groups(ConnTables& t, const std::vector<std::vector<Term>>* per_group) {
  const size_t ng = t.groups.size();
  std::vector<uint64_t> gkey(ng);
  t.max_lowered = 0;
  for (size_t g = 0; g < ng; ++g) {
    int low[kMaxOrder], r = 0;
    for (int k = 0; k < t.groups[g].nchg; ++k)
      if (t.groups[g].delta[k] < 0) low[r++] = t.groups[g].mode[k];  // modes are ascending
    gkey[g] = lowered_key(r, low);
    t.max_lowered = std::max(t.max_lowered, r);
  }
  std::vector<size_t> ord(ng);
  for (size_t g = 0; g < ng; ++g) ord[g] = g;
  std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return gkey[a] < gkey[b]; });
  std::vector<Group> sorted(ng);
  t.seg_key.clear();
  t.seg_begin.clear();
  for (size_t i = 0; i < ng; ++i) {
    const size_t g = ord[i];
    sorted[i] = t.groups[g];
    if (t.seg_key.empty() || t.seg_key.back() != gkey[g]) {
      t.seg_key.push_back(gkey[g]);
      t.seg_begin.push_back((int)i);
    }
    sorted[i].term_begin = (int)t.terms.size();
    if (per_group) t.terms.insert(t.terms.end(), (*per_group)[g].begin(), (*per_group)[g].end());
    sorted[i].term_end = (int)t.terms.size();
  }
  t.seg_begin.push_back((int)ng);
  t.groups.swap(sorted);
}

void build_conn_tables(const Model& m, ConnTables& t) {
  t.groups.clear(); t.terms.clear(); t.diag_terms.clear();
  std::map<std::vector<int>, int> index;         // change vector -> group id
  std::vector<std::vector<Term>> per_group;
  // summation order of the reference's pair loops: quartic, sextic | cubic, quintic
  const int order_seq[4] = {4, 6, 3, 5};
  for (int oi = 0; oi < 4; ++oi)
    for (const auto& f : m.fcs) {
      if (f.order != order_seq[oi]) continue;
      for_each_pattern(f.nk, f.powers, [&](const int* d) {
        int qd = 0, mc = 0;
        for (int k = 0; k < f.nk; ++k) { qd += std::abs(d[k]); mc += d[k] != 0; }
        bool ok = (qd % 2 == 0) ? (qd <= m.fcmax && mc <= m.fcmax)
                                : (qd <= m.fcmax - 1 && mc <= m.fcmax - 1);
        if (!ok) return;
        Term tm{};
        tm.fc = f.fc;
        tm.nk = (uint8_t)f.nk;
        for (int k = 0; k < f.nk; ++k) {
          tm.mode[k] = (uint8_t)f.modes[k];
          tm.pw[k] = (uint8_t)f.powers[k];
          tm.dl[k] = (int8_t)d[k];
        }
        if (qd == 0) { t.diag_terms.push_back(tm); return; }
        std::vector<std::pair<int, int>> chg;
        for (int k = 0; k < f.nk; ++k)
          if (d[k]) chg.push_back({f.modes[k], d[k]});
        std::sort(chg.begin(), chg.end());
        std::vector<int> key;
        for (auto& c : chg) { key.push_back(c.first); key.push_back(c.second); }
        auto it = index.find(key);
        int gid;
        if (it == index.end()) {
          gid = (int)per_group.size();
          index.emplace(key, gid);
          per_group.emplace_back();
          Group g;
          g.nchg = (int)chg.size();
          for (int k = 0; k < g.nchg; ++k) { g.mode[k] = chg[k].first; g.delta[k] = chg[k].second; }
          t.groups.push_back(g);
        } else {
          gid = it->second;
        }
        per_group[gid].push_back(tm);
      });
    }
  index_groups(t, &per_group);
}

bool build_gate_patterns(const Model& m, ConnTables& t, int64_t max_patterns) {
  t.groups.clear(); t.terms.clear(); t.diag_terms.clear();
  const int nm = m.nm;
  // change vectors with |delta|_1 = s, s even <= fcmax or s odd <= fcmax - 1 (Ham.cpp:247,283);
  // the number of changed modes is at most s, so the mode-count gates hold by themselves
  const int smax = m.fcmax;
  std::vector<int> modes(kMaxOrder), deltas(kMaxOrder);
  bool over = false;
  // choose k modes m_1 < .. < m_k and nonzero deltas with sum |d| = s
  std::function<void(int, int, int, int)> rec = [&](int start, int k, int used, int s) {
    if (over) return;
    if (used == s) {
      if (k == 0) return;
      Group g;
      g.nchg = k;
      for (int a = 0; a < k; ++a) { g.mode[a] = modes[a]; g.delta[a] = deltas[a]; }
      t.groups.push_back(g);
      if ((int64_t)t.groups.size() > max_patterns) over = true;
      return;
    }
    if (k == kMaxOrder) return;
    for (int mm = start; mm < nm; ++mm)
      for (int d = 1; used + d <= s; ++d)
        for (int sg = -1; sg <= 1; sg += 2) {
          modes[k] = mm;
          deltas[k] = sg * d;
          rec(mm + 1, k + 1, used + d, s);
          if (over) return;
        }
  };
  for (int s = 1; s <= smax && !over; ++s) {
    if (s % 2 == 1 && s > smax - 1) continue;
    rec(0, 0, 0, s);
  }
  if (over) { t.groups.clear(); return false; }
  index_groups(t, nullptr);
  return true;
}

void build_hb_entries(const Model& m, std::vector<HBEntry>& e, std::vector<int64_t>& cum) {
  e.clear();
  cum.assign(1, 0);
  for (const auto& f : m.hb) {
    HBEntry h{};
    h.fc = f.fc;
    h.absfc = std::fabs(f.fc);
    h.nk = f.nk;
    int total = 1;
    bool all_even = true;
    for (int k = 0; k < f.nk; ++k) {
      h.modes[k] = f.modes[k];
      h.powers[k] = f.powers[k];
      total *= f.powers[k] + 1;
      if (f.powers[k] % 2) all_even = false;
    }
    h.zero_idx = -1;
    if (all_even) {
      int idx = 0;
      for (int k = 0; k < f.nk; ++k) idx = idx * (f.powers[k] + 1) + f.powers[k] / 2;
      h.zero_idx = idx;
    }
    h.npat = total - (all_even ? 1 : 0);
    e.push_back(h);
    cum.push_back(cum.back() + h.npat);
  }
}

double ladder_ref(int p, int n, int d) {
  // Ham.cpp:38-104: expand (a + a^dag)^p applied to |n>, creation branch first at each step,
  // then sum the coefficients of the paths that end on |n+d>.
  std::vector<int> st{n};
  std::vector<double> co{1.0};
  for (int j = 0; j < p; ++j) {
    std::vector<int> s2;
    std::vector<double> c2;
    for (size_t k = 0; k < st.size(); ++k) {
      int q = st[k];
      s2.push_back(q + 1);
      c2.push_back(co[k] * std::sqrt(q + 1));
      if (q - 1 >= 0) {
        s2.push_back(q - 1);
        c2.push_back(co[k] * std::sqrt(q));
      }
    }
    st.swap(s2);
    co.swap(c2);
  }
  double s = 0.0;
  for (size_t k = 0; k < st.size(); ++k)
    if (st[k] == n + d) s += co[k];
  return s;
}

void ladder_table(int qmax, std::vector<double>& T) {
  T.assign((size_t)(kMaxOrder + 1) * (qmax + 1) * 13, 0.0);
  for (int p = 1; p <= kMaxOrder; ++p)
    for (int q = 0; q <= qmax; ++q)
      for (int d = -p; d <= p; ++d) {
        if (q + d < 0) continue;
        int lo = std::min(q, q + d);
        T[((size_t)p * (qmax + 1) + q) * 13 + d + 6] = ladder_ref(p, lo, std::abs(d));
      }
}

double harmonic_energy(const Model& m, const uint8_t* q) {
  double e = 0.;
  for (int j = 0; j < m.nm; ++j) {
    double ej = 0.5;
    ej += q[j];
    ej *= m.freq[j];
    e += ej;
  }
  return e;
}

}  // namespace vhci
