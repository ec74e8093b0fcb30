// `vhci` command-line tool: drop-in for the reference's `vhci -n Ncpus -i in.inp -o freqs.dat
// [-c checkpoint]` (VHCI.cpp:5-185, Input_Reader.cpp:17-168) on top of the C ABI.  stdout carries
// the reference's messages; handled errors exit with status 0 as the reference does, unless
// --strict is given (then 1).  Extra flags: --mixed (FP32 Hamiltonian storage), --device N,
// --stored-sparsity (the "% sparse" line from the stored nonzero entries instead of the
// reference's structural pattern count).
#include <sys/stat.h>

#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>

#include "vhci_gpu.h"

namespace {

bool strict = false;

[[noreturn]] void quit() { std::exit(strict ? 1 : 0); }

void banner() {
  std::cout << '\n';
  std::cout << "######################################" << "#######################################" << '\n';
  std::cout << "#                                       " << "                                    #" << '\n';
  std::cout << "#              " << "Vibrational Heat-Bath Configuration Interaction" << "              #" << '\n';
  std::cout << "#                         " << "By: Jonathan H. Fetherolf" << "                         #" << '\n';
  std::cout << "#                                       " << "                                    #" << '\n';
  std::cout << "#                      " << "Based on LOVCI by Eric G. Kratz" << "                      #" << '\n';
  std::cout << "#                                       " << "                                    #" << '\n';
  std::cout << "######################################" << "#######################################" << '\n' << '\n';
  std::cout.flush();
}

void usage_short() {
  std::cout << "Usage: vhci -n Ncpus -i Modes.inp -o Freqs.dat -c Checkpoint.txt";
  std::cout << '\n' << '\n' << "Use -h or --help for detailed instructions." << '\n' << '\n';
  std::cout.flush();
}

void print_time(const char* label, int t0) {
  double rt = (double)((unsigned)time(0) - t0);
  std::string unit = "seconds";
  if (rt >= 3600) { rt /= 3600; unit = "hours"; }
  else if (rt >= 60) { rt /= 60; unit = "minutes"; }
  std::cout << std::fixed << std::setprecision(2) << label << rt << " " << unit;
}

std::string err_of(vhci_ctx* c) {
  char b[512] = {0};
  if (c) vhci_last_error(c, b, sizeof b);
  return b;
}

[[noreturn]] void die(vhci_ctx* c, int st) {
  std::string e = err_of(c);
  if (e.empty()) e = "error code " + std::to_string(st);
  std::cout << e << std::endl;
  vhci_destroy(c);
  quit();
}

}  // namespace

int main(int argc, char* argv[]) {
  const int start = (unsigned)time(0);
  std::cout.precision(12);
  std::cout << std::fixed;
  banner();
  std::cout << "Reading input..." << '\n';
  // extra flags are stripped before the reference's argument rules apply
  vhci_opts o;
  vhci_default_opts(&o);
  o.verbose = 1;
  o.structural_nnz = 1;  // the reference's "% sparse" counts structural zeros too
  std::string inp, outp, cp = "none";
  int ncpus = 0;
  bool have_in = false, have_out = false;
  std::vector<std::string> args;
  for (int i = 0; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "--strict") { strict = true; continue; }
    if (a == "--mixed") { o.precision = 1; continue; }
    if (a == "--stored-sparsity") { o.structural_nnz = 0; continue; }
    if (a == "--device" && i + 1 < argc) { o.device = std::atoi(argv[++i]); continue; }
    args.push_back(a);
  }
  const int ac = (int)args.size();
  if (ac == 1) {
    std::cout << '\n' << "Missing arguments..." << '\n' << '\n';
    usage_short();
    quit();
  }
  if ((ac % 2) != 1 && args[1] != "-h" && args[1] != "--help") {
    std::cout << '\n' << "Wrong number of arguments..." << '\n' << '\n';
    usage_short();
    quit();
  }
  for (int i = 0; i < ac; ++i) {
    const std::string& a = args[i];
    if (a == "-h" || a == "--help") {
      std::cout << '\n' << "Usage: vhci -n Ncpus -i Modes.inp -o Freqs.txt" << '\n' << '\n';
      std::cout << "Command line arguments:" << '\n' << '\n';
      std::cout << "  -n    Number of CPUs to use for the calculation." << '\n' << '\n';
      std::cout << "  -i    Input file." << '\n' << '\n';
      std::cout << "  -o    Output file for the first NEig VCI frequencies." << '\n' << '\n';
      std::cout << "  -c    Checkpoint file for HCI iterations on large systems." << '\n' << '\n';
      std::cout.flush();
      quit();
    }
    if (i + 1 >= ac) break;
    if (a == "-n") ncpus = std::atoi(args[i + 1].c_str());
    if (a == "-i") { inp = args[i + 1]; have_in = true; }
    if (a == "-o") { outp = args[i + 1]; have_out = true; }
    if (a == "-c") cp = args[i + 1];
  }
  const int maxt = (int)std::max(1u, std::thread::hardware_concurrency());
  if (ncpus < 1) {
    std::cout << " Warning: Calculations cannot run with " << ncpus << " CPUs." << '\n';
    std::cout << "  Do you know how computers work?" << " Ncpus set to 1" << '\n';
    ncpus = 1;
  }
  if (ncpus > maxt) {
    std::cout << " Warning: Too many threads requested." << '\n';
    std::cout << "  Requested: " << ncpus << "," << " Available: " << maxt << '\n';
    std::cout << "  Ncpus set to " << maxt << '\n';
    ncpus = maxt;
  }
  o.host_threads = ncpus;
  bool doquit = false;
  {
    std::ifstream t(inp);
    if (!have_in || !t.good()) { std::cout << " Error: Could not open input file." << '\n'; doquit = true; }
  }
  {
    std::ofstream t;
    if (have_out) t.open(outp, std::ios_base::out);
    if (!have_out || !t.good()) { std::cout << " Error: Could not output file." << '\n'; doquit = true; }
  }
  if (doquit) { std::cout << '\n'; std::cout.flush(); quit(); }
  std::cout << '\n' << "No fatal errors detected." << '\n' << " And there was much rejoicing. Yay..." << '\n' << '\n';
  int restart = 0;
  if (cp == "none") {
    std::cout << "No checkpoint filename specified. Checkpoints will not be saved." << '\n' << '\n';
  } else {
    std::cout << "Locating checkpoint file..." << '\n';
    std::ifstream t(cp);
    restart = (t.good() && t.peek() != std::ifstream::traits_type::eof()) ? 1 : 0;
    if (restart) std::cout << "Checkpoint file found. Calculation will be resumed." << '\n' << '\n';
    else std::cout << "No checkpoint file found. Calculation will start from the beginning." << '\n' << '\n';
  }
  std::cout.flush();

  vhci_ctx* c = nullptr;
  int st = vhci_create_from_file(inp.c_str(), &o, restart, &c);
  if (st != VHCI_OK) die(c, st);
  vhci_info info;
  vhci_get_info(c, &info);
  std::cout << "General settings:" << '\n';
  std::cout << "  CPU threads: " << ncpus << '\n' << '\n';
  std::cout << "  Normal modes: " << info.nmodes << '\n';
  {
    std::ifstream t(inp);
    std::string line, tok;
    std::getline(t, line);
    double d;
    int ntot = 0;
    t >> tok >> d >> tok >> d >> tok >> d >> tok >> d >> tok >> ntot;
    std::cout << "  Max quanta per state: " << ntot << '\n';
  }
  std::cout << "  Basis functions: " << info.n_basis << '\n';
  std::cout << "  Force constants: ";
  if (info.n_fc == 0) std::cout << "N/A" << '\n' << '\n';
  else std::cout << info.n_fc << '\n' << '\n';
  if (info.eps1 != 0.) {
    std::cout << std::setprecision(3) << "  Using HCI with energy cutoff: " << info.eps1 << '\n';
    if (info.nstate == 1) std::cout << "  Optimizing just the ground states (ZPE)." << '\n';
    else std::cout << "  Optimizing the first " << info.nstate << " eigenstates." << '\n';
  }
  std::cout << '\n';
  std::cout.precision(12);
  std::cout.flush();

  if (restart) {
    std::cout << '\n' << "Loading checkpoint file...";
    std::cout.flush();
    st = vhci_read_checkpoint(c, cp.c_str());
    if (st != VHCI_OK) die(c, st);
    std::cout << "done." << '\n';
    vhci_get_info(c, &info);
    std::cout << "  Basis functions: " << info.n_basis << '\n' << std::endl;
  }
  if (info.eps1 != 0.) std::cout << "Beginning Heat Bath CI procedure..." << '\n';
  st = vhci_hci(c, cp == "none" ? nullptr : cp.c_str(), nullptr, nullptr);
  if (st != VHCI_OK) die(c, st);
  if (info.pt2) {
    print_time(" Variational stage took ", start);
    std::cout << '\n' << '\n';
    std::cout << "Performing Epstein-Nesbet perturbation theory..." << std::endl;
    if (info.eps2 > 0)
      std::cout << " Using heat bath sorting of perturbative states with cutoff: " << std::scientific
                << info.eps2 << std::fixed << std::endl;
    else
      std::cout << " Including all connected states in PT2 calculation." << std::endl;
    int64_t np = 0;
    st = vhci_pt2(c, info.eps2, nullptr, &np);
    if (st != VHCI_OK) die(c, st);
  }
  std::cout.precision(10);
  st = vhci_write_freqs(c, outp.c_str());
  if (st != VHCI_OK) die(c, st);
  double E[1] = {0};
  int ne = 0;
  vhci_get_energies(c, E, 1, &ne);
  // ZPE = smallest held eigenvalue (VHCI.cpp:122); eigenvalues are not re-sorted after PT2
  std::vector<double> all(info.nstate);
  vhci_get_energies(c, all.data(), info.nstate, &ne);
  double zpe = all[0];
  for (int i = 1; i < ne; ++i) zpe = std::min(zpe, all[i]);
  if (zpe < 0) {
    std::cout << "Error: The zero-point energy is negative." << " Something is wrong." << '\n';
    std::cout << "Try reducing the number of quanta or removing" << " large anharmonic" << '\n';
    std::cout << "force constants." << '\n' << '\n';
    std::cout.flush();
    vhci_destroy(c);
    quit();
  }
  std::cout << "Printing the results..." << '\n' << '\n' << "Results:" << '\n';
  std::cout << "  Zero-point energy: " << std::setprecision(2) << zpe << " (1/cm)" << '\n';
  print_time("  Run time: ", start);
  std::cout << '\n' << '\n' << "Done." << '\n' << '\n';
  std::cout.flush();
  vhci_destroy(c);
  return 0;
}
