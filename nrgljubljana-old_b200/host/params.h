// `param` file ([param] block of key=value lines, src/misc.h:71-124) and the
// subset of the reference's parameters (src/param.cc:95-582) that the NRG
// iteration hot path uses, with the reference's defaults.
#pragma once
#include <map>
#include <string>

namespace nrgb {

struct Params {
  double Lambda = 1.0, z = 1.0, bandrescale = 1.0;
  std::string discretization = "Y";
  int Ninit = 0, Nmax = 0;
  int keep = 100, keepmin = 0;
  double keepenergy = -1.0;
  double safeguard = 1e-5;
  int safeguardmax = 200;
  double fixeps = 1e-15;
  double betabar = 1.0, T = -999.0;
  std::string strategy = "kept";
  bool lastall = false, lastalloverride = false;
  bool dm = false, dmnrg = false, fdm = false, cfs = false;
  std::string specd, spect, specs;
  int bins = 100;
  double emin = -1.0, emax = -1.0, goodE = 2.0;
  bool NN1 = false, NN2even = true, NN2avg = false;
  double NNtanh = 0.0;
  double discard_trim = 1e-16, discard_immediately = 1e-16;
  bool savebins = false, broaden = true;
  double broaden_max = 2.5, broaden_min = -99.0, broaden_min_ratio = 3.0, broaden_ratio = 1.05;
  double alpha = 0.3, omega0 = -1.0, omega0_ratio = 1.0;
  int dumpannotated = 0, dumpprecision = 8;
  bool dumpscaled = true, dumpabs = false, dumpgroups = true;
  double grouptol = 1e-6;
  int width_td = 16, prec_td = 10, width_custom = 16, prec_custom = 10, prec_xy = 10;
  bool calc0 = true;  // td/custom/annotated rows of the initial cluster (src/param.cc:490)
  // Products of the recalculation, density matrices and spectral weights:
  // 0 = FP64 on the FP64 tensor pipe; 2..8 = split precision with this many
  // INT8 slices per operand (this implementation's key; the reference has
  // no such parameter and reports it as unknown).
  int gemm_slices = 0;
  // Transformation files (src/dmnrg.h:183-304, src/nrg.cc:3512-3524): with
  // removefiles=false every step's eigen-decompositions are written to
  // <workdir>/unitary<N>; with resume=true the steps that have such a file
  // load it instead of diagonalising.  The file layout is this
  // implementation's own (the reference writes boost archives).
  bool removefiles = true, resume = false;
  int channels = 1;  // from the data file

  // Parse `path`; unknown keys are kept in `unused` (the reference reports them).
  void read(const std::string& path);
  std::map<std::string, std::string> unused;
};

// SCALE(N) of src/nrg.cc:491-506 (no substeps).
double scale_of(const Params& P, int N);

}  // namespace nrgb
