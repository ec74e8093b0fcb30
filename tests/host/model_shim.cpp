// Test shim over the host-side model code (vhci_b200/csrc/model.cpp), built by tests/test_model_host.py
// with g++ alone: exposes the connection-group and gate-pattern tables so their ordering and
// segment index can be checked on the CPU.
#include <cstring>

#include "model.h"

using namespace vhci;

namespace {
Model g_model;
ConnTables g_tab;
}

extern "C" {

// 0 on success; which = 0: connection groups, 1: gate patterns (limit max_patterns).
int shim_load(const char* path, int which, long long max_patterns) {
  std::string err;
  g_model = Model();
  if (!parse_input_file(path, g_model, err)) return 1;
  if (!finalize_model(g_model, false, err)) return 2;
  if (which == 0) build_conn_tables(g_model, g_tab);
  else if (!build_gate_patterns(g_model, g_tab, max_patterns)) return 3;
  return 0;
}

long long shim_ngroups() { return (long long)g_tab.groups.size(); }
long long shim_nseg() { return (long long)g_tab.seg_key.size(); }
int shim_max_lowered() { return g_tab.max_lowered; }
int shim_fcmax() { return g_model.fcmax; }
int shim_nm() { return g_model.nm; }

// group u: nchg, then (mode, delta) pairs into out[0..2*nchg)
int shim_group(long long u, int* out) {
  const Group& g = g_tab.groups[(size_t)u];
  for (int k = 0; k < g.nchg; ++k) { out[2 * k] = g.mode[k]; out[2 * k + 1] = g.delta[k]; }
  return g.nchg;
}

unsigned long long shim_seg_key(long long s) { return g_tab.seg_key[(size_t)s]; }
long long shim_seg_begin(long long s) { return g_tab.seg_begin[(size_t)s]; }
unsigned long long shim_lowered_key(int r, const int* modes) { return lowered_key(r, modes); }
}
