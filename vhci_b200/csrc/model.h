// Host-side problem model: the parsed input, scaled force constants, heat-bath list, initial
// basis, the connection-group tables that replace the reference's pair screening, and the
// harmonic-oscillator ladder-factor table.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "vhci_gpu.h"

namespace vhci {

constexpr int kMaxOrder = 6;

struct ForceConstant {
  double fc = 0.0;            // scaled value (raw * 1/sqrt(2^order) / prod p_k!)
  int order = 0;              // number of mode indices (fcpow.size() in the reference)
  int nk = 0;                 // distinct modes
  int modes[kMaxOrder] = {};  // distinct modes in first-appearance order (ShortModes)
  int powers[kMaxOrder] = {}; // power per distinct mode (ModePowers)
};

struct Model {
  int nm = 0, ntot = 0, nstate = 0, pt2 = 0;
  double eps1 = 0.0, eps2 = 0.0;
  int nfc_in = 0;
  std::vector<double> freq;
  std::vector<int> cap;
  std::vector<ForceConstant> fcs;  // input order, scaled
  std::vector<ForceConstant> hb;   // heat-bath list, |fc| descending
  int fcmax = 0;                   // largest FC order present
  std::vector<uint8_t> init_basis; // n0 x nm quanta, reference enumeration order
  int64_t n0 = 0;
};

// Positional parse with the reference's rules; fills raw values (unscaled).  On failure returns
// false and a message in the reference's wording.
bool parse_input_file(const char* path, Model& m, std::string& err);
bool model_from_problem(const vhci_problem* p, Model& m, std::string& err);
// Scale FCs, check orders, build the heat-bath list and the initial basis.
bool finalize_model(Model& m, bool restart, std::string& err);

// ---- connection groups (Hamiltonian build and PT2) ----
// Every FC pattern (delta_k in {-p_k, -p_k+2, .., p_k} on its modes) moves a state by a fixed
// quanta change.  Patterns of all FCs with the same change vector form one group; a state is
// connected to state+change by the sum of the group's terms.  The Delta=0 group holds the
// diagonal terms.  Patterns refused by the reference's pair gate (odd change with
// qdiff > fcmax-1 or mchange > fcmax-1, Ham.cpp:283) are left out.
struct Term {
  double fc;
  uint8_t nk;
  uint8_t mode[kMaxOrder];
  uint8_t pw[kMaxOrder];
  int8_t dl[kMaxOrder];
};

struct Group {
  int nchg = 0;
  int mode[kMaxOrder] = {};
  int delta[kMaxOrder] = {};
  int term_begin = 0, term_end = 0;
};

// Key of the set of modes a change vector lowers (delta < 0), modes ascending:
// (r + 1) | sum_i (mode_i + 1) << (3 + 7 i), r <= 6 lowered modes, modes < 127.
inline uint64_t lowered_key(int r, const int* modes_ascending) {
  uint64_t key = (uint64_t)(r + 1);
  for (int i = 0; i < r; ++i) key |= (uint64_t)(modes_ascending[i] + 1) << (3 + 7 * i);
  return key;
}

// Groups are ordered by the key of their lowered-mode set, so the groups that lower one mode set
// form one segment.  A state can only move by a group whose lowered modes are all excited in it;
// enumerating the subsets of a state's excited modes and visiting their segments skips every
// group that lowers an unexcited mode.
struct ConnTables {
  std::vector<Group> groups;     // off-diagonal groups, ordered by lowered-mode key
  std::vector<Term> terms;       // terms of the off-diagonal groups, contiguous per group
  std::vector<Term> diag_terms;  // Delta = 0 terms (quartic then sextic, input order)
  std::vector<uint64_t> seg_key; // lowered-mode key of each segment (ascending)
  std::vector<int> seg_begin;    // first group of each segment, plus the end
  int max_lowered = 0;           // most modes one group lowers
};
void build_conn_tables(const Model& m, ConnTables& t);
// Every change vector the reference's pair gates admit (|delta|_1 = s, s even <= fcmax, s odd <=
// fcmax - 1; Ham.cpp:247,283), as groups without terms, indexed like the connection groups.
// False (and empty) when there are more than max_patterns.
bool build_gate_patterns(const Model& m, ConnTables& t, int64_t max_patterns);

// ---- heat-bath pattern descriptors ----
struct HBEntry {
  double fc;      // signed scaled value
  double absfc;   // |fc|
  int nk;
  int modes[kMaxOrder];
  int powers[kMaxOrder];
  int npat;       // patterns excluding the all-zero one
  int zero_idx;   // mixed-radix index of the all-zero pattern, -1 if none
};
void build_hb_entries(const Model& m, std::vector<HBEntry>& e, std::vector<int64_t>& cum);

// ---- ladder factors ----
// <n+d| (a + a^dag)^p |n> by the reference's path expansion (Ham.cpp:38-104), for p <= 6.
double ladder_ref(int p, int n, int d);
// Table Tc[(p * (qmax+1) + q) * 13 + d + 6] = ladder_ref(p, min(q, q+d), |d|) (0 when q+d < 0):
// the factor is taken from the lower state, so H_ij and H_ji are the same bits.
void ladder_table(int qmax, std::vector<double>& T);

// Harmonic energy in the reference's operation order (Ham.cpp:211-220).
double harmonic_energy(const Model& m, const uint8_t* q);

}  // namespace vhci
