#include "params.h"

#include <math.h>

#include <fstream>
#include <stdexcept>

namespace nrgb {

namespace {
bool as_bool(const std::string& s) { return s == "true" || s == "1" || s == "yes" || s == "True"; }
std::string rstrip(std::string s) {
  while (!s.empty() && (s.back() == ' ' || s.back() == '\t' || s.back() == '\r')) s.pop_back();
  return s;
}
}  // namespace

void Params::read(const std::string& path) {
  std::ifstream F(path);
  if (!F) throw std::runtime_error("Can't open " + path + " for reading.");
  std::string line;
  bool inblock = false;
  std::map<std::string, std::string> kv;
  while (std::getline(F, line)) {
    if (!inblock) {
      if (rstrip(line) == "[param]") inblock = true;
      continue;
    }
    if (!line.empty() && line[0] == '[') break;
    const auto eq = line.find('=');
    if (eq == std::string::npos) continue;
    const std::string key = line.substr(0, eq);
    if (kv.count(key)) throw std::runtime_error("Duplicate keyword: " + key);
    kv[key] = rstrip(line.substr(eq + 1));
  }
  auto D = [&](const char* k, double& v) { if (kv.count(k)) { v = std::stod(kv[k]); kv.erase(k); } };
  auto I = [&](const char* k, int& v) { if (kv.count(k)) { v = (int)std::stod(kv[k]); kv.erase(k); } };
  auto B = [&](const char* k, bool& v) { if (kv.count(k)) { v = as_bool(kv[k]); kv.erase(k); } };
  auto S = [&](const char* k, std::string& v) { if (kv.count(k)) { v = kv[k]; kv.erase(k); } };
  D("Lambda", Lambda); D("z", z); D("bandrescale", bandrescale); S("discretization", discretization);
  I("Ninit", Ninit); I("Nmax", Nmax); I("keep", keep); I("keepmin", keepmin); D("keepenergy", keepenergy);
  D("safeguard", safeguard); I("safeguardmax", safeguardmax); D("fixeps", fixeps);
  D("betabar", betabar); D("T", T); S("strategy", strategy);
  B("lastall", lastall); B("lastalloverride", lastalloverride);
  B("dm", dm); B("dmnrg", dmnrg); B("fdm", fdm); B("cfs", cfs);
  S("specd", specd); S("spect", spect); S("specs", specs);
  I("bins", bins); D("emin", emin); D("emax", emax); D("goodE", goodE);
  B("NN1", NN1); B("NN2even", NN2even); B("NN2avg", NN2avg); D("NNtanh", NNtanh);
  D("discard_trim", discard_trim); D("discard_immediately", discard_immediately);
  B("savebins", savebins); B("broaden", broaden); D("broaden_max", broaden_max);
  D("broaden_min", broaden_min); D("broaden_min_ratio", broaden_min_ratio); D("broaden_ratio", broaden_ratio);
  D("alpha", alpha); D("omega0", omega0); D("omega0_ratio", omega0_ratio);
  I("dumpannotated", dumpannotated); I("dumpprecision", dumpprecision); B("dumpscaled", dumpscaled);
  B("dumpabs", dumpabs); B("dumpgroups", dumpgroups); D("grouptol", grouptol);
  I("width_td", width_td); I("prec_td", prec_td); I("width_custom", width_custom);
  I("prec_custom", prec_custom); I("prec_xy", prec_xy);
  B("calc0", calc0);
  I("gemm_slices", gemm_slices);
  B("removefiles", removefiles);
  B("resume", resume);
  unused = kv;
  // validateparameters (src/read-input.cc:6-36) and calculate_invariants
  if (keep <= 1) throw std::runtime_error("keep must be > 1");
  if (gemm_slices != 0 && (gemm_slices < 2 || gemm_slices > 8))
    throw std::runtime_error("gemm_slices must be 0 (FP64) or in [2, 8]");
  if (Lambda <= 1.0) throw std::runtime_error("Lambda must be > 1");
  if (dmnrg || fdm || cfs) dm = true;
  if ((fdm || cfs) && !lastalloverride) lastall = true;
  discretization = discretization.substr(0, 1);
}

double scale_of(const Params& P, int N) {
  double s = 0.0;
  if (P.discretization == "Y") s = 0.5 * (1.0 + 1.0 / P.Lambda);
  if (P.discretization == "C" || P.discretization == "Z") s = (1.0 - 1.0 / P.Lambda) / log(P.Lambda);
  s *= pow(P.Lambda, -(N - 1) / 2.0 + 1.0 - P.z);
  if (s == 0.0) throw std::runtime_error("unknown discretization " + P.discretization);
  return s * P.bandrescale;
}

}  // namespace nrgb
