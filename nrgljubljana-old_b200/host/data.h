// The `data` input file, version 9 (writer: initial.m:4094-4392; reader:
// src/nrg.cc:3293-3401 and src/read-input.cc:39-143): header with the
// symmetry type, channels / chain length / subspace count, initial
// eigenenergies per invariant subspace, <I1||f^dag||I2> blocks per channel,
// the ground-state energy, operator blocks (s, p, g, d, t, o, q + name) and
// the Wilson-chain coefficient tables (z: xi, zeta per channel).
#pragma once
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace nrgb {

using Invar = std::pair<int, int>;          // (Q, SS) for QS, (Q, SSZ) for QSZ, (0, SS) for SPSU2
using Twoinvar = std::pair<Invar, Invar>;   // (bra, ket) subspaces

struct HostMat {
  int rows = 0, cols = 0;
  std::vector<double> a;  // column-major
};

using HostBlocks = std::map<Twoinvar, HostMat>;

struct DataFile {
  std::string symtype;
  int channels = 0, Nmax = 0;
  std::map<Invar, std::vector<double>> energies;
  std::vector<HostBlocks> opch;                                // one per channel
  double gs_energy = 0.0;
  std::map<char, std::map<std::string, HostBlocks>> ops;       // kind -> name -> blocks
  std::vector<std::vector<double>> xi, zeta;                   // per channel, index 0..Nmax
  // superconducting baths (block Z, src/nrg.cc:3383-3386): on-site pairing
  // delta and anomalous hopping kappa per channel; empty when absent
  std::vector<std::vector<double>> delta, kappa;

  // Entry n of table t for channel ch, 0 where the file has no such table.
  static double chain_coef(const std::vector<std::vector<double>>& t, int ch, int n) {
    if (ch >= (int)t.size()) return 0.0;
    if (n < 0 || n >= (int)t[ch].size()) throw std::runtime_error("chain coefficient index out of range");
    return t[ch][n];
  }

  void read(const std::string& path);
};

}  // namespace nrgb
