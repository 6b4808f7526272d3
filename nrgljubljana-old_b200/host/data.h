// The `data` input file, version 9 (writer: initial.m:4094-4392; reader:
// src/nrg.cc:3293-3401 and src/read-input.cc:39-143): header with the
// symmetry type, channels / chain length / subspace count, initial
// eigenenergies per invariant subspace, <I1||f^dag||I2> blocks per channel,
// the ground-state energy, operator blocks (s, p, g, d, t, o, q + name) and
// the Wilson-chain coefficient tables (z: xi, zeta per channel).
#pragma once
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace nrgb {

using Invar = std::pair<int, int>;          // (Q, SS) for the QS symmetry
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

  void read(const std::string& path);
};

}  // namespace nrgb
