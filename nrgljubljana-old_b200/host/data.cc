#include "data.h"

#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace nrgb {

namespace {

// Token stream over the lines of the file that skips '#' comment lines.
struct Tokens {
  std::vector<std::string> lines;
  size_t line = 0;
  std::istringstream cur;
  bool have = false;

  bool next(std::string& t) {
    while (true) {
      if (have && (cur >> t)) return true;
      if (line >= lines.size()) return false;
      const std::string& l = lines[line++];
      size_t p = l.find_first_not_of(" \t\r");
      if (p != std::string::npos && l[p] == '#') continue;
      cur.clear();
      cur.str(l);
      have = true;
    }
  }
  std::string tok() {
    std::string t;
    if (!next(t)) throw std::runtime_error("data file ended early");
    return t;
  }
  int i() { return std::stoi(tok()); }
  double d() {
    const double x = std::stod(tok());
    if (!std::isfinite(x)) throw std::runtime_error("data file: value not finite");
    return x;
  }
};

}  // namespace

void DataFile::read(const std::string& path) {
  std::ifstream F(path);
  if (!F) throw std::runtime_error("Can't load initial data.");
  Tokens T;
  std::string l;
  while (std::getline(F, l)) T.lines.push_back(l);
  int version = -1;
  size_t pos = 0;
  while (pos < T.lines.size() && !T.lines[pos].empty() && T.lines[pos][0] == '#') {
    const std::string& h = T.lines[pos];
    if (h.size() > 1 && h[1] == '!') version = std::stoi(h.substr(2));
    else if (h.find("symtype", 1) != std::string::npos) {
      const auto p = h.find_last_of(" \t");
      if (p != std::string::npos && p + 1 < h.size()) symtype = h.substr(p + 1);
    }
    ++pos;
  }
  if (version != 9) throw std::runtime_error("data file version mismatch (expected 9)");
  T.line = pos;
  // invariants are written with one integer per quantum number: SPSU2 has
  // the spin alone (read as (0, SS))
  const bool one_qn = symtype == "SPSU2";
  auto read_invar = [&](Invar& I) {
    I.first = one_qn ? 0 : T.i();
    I.second = T.i();
  };
  channels = T.i();
  Nmax = T.i();
  const int nsubs = T.i();
  if (nsubs <= 0) throw std::runtime_error("data file: no subspaces");
  for (int s = 0; s < nsubs; ++s) {
    Invar I;
    read_invar(I);
    const int n = T.i();
    if (n <= 0) throw std::runtime_error("data file: empty subspace");
    std::vector<double> e(n);
    for (auto& x : e) x = T.d();
    energies[I] = e;
  }
  auto read_blocks = [&](HostBlocks& b) {
    const int nf = T.i();
    for (int k = 0; k < nf; ++k) {
      Invar I1, I2;
      read_invar(I1);
      read_invar(I2);
      HostMat M;
      M.rows = energies.count(I1) ? (int)energies[I1].size() : 0;
      M.cols = energies.count(I2) ? (int)energies[I2].size() : 0;
      M.a.assign((size_t)M.rows * M.cols, 0.0);
      for (int r = 0; r < M.rows; ++r)      // rows are written one per line
        for (int c = 0; c < M.cols; ++c) M.a[r + (size_t)c * M.rows] = T.d();
      b[{I1, I2}] = std::move(M);
    }
  };
  opch.resize(channels);
  for (int ch = 0; ch < channels; ++ch) {
    const std::string f = T.tok();
    const int i = T.i(), j = T.i();
    if (f != "f" || i != ch || j != 0) throw std::runtime_error("data file: bad f block header");
    read_blocks(opch[ch]);
  }
  // operator / table blocks, each introduced by a line "<kind><name>"
  T.have = false;
  while (T.line < T.lines.size()) {
    std::string h = T.lines[T.line++];
    const size_t p = h.find_first_not_of(" \t\r");
    if (p == std::string::npos) continue;
    h = h.substr(p);
    while (!h.empty() && (h.back() == '\r' || h.back() == ' ' || h.back() == '\t')) h.pop_back();
    const char kind = h[0];
    const std::string name = h.substr(1);
    if (kind == '#') continue;
    if (kind == 'e') {
      gs_energy = T.d();
    } else if (kind == 's' || kind == 'p' || kind == 'g' || kind == 'd' || kind == 't' ||
               kind == 'o' || kind == 'q') {
      read_blocks(ops[kind][name]);
    } else if (kind == 'z' || kind == 'Z') {
      // z: xi then zeta; Z: delta then kappa; one table per channel each
      auto& t1 = kind == 'z' ? xi : delta;
      auto& t2 = kind == 'z' ? zeta : kappa;
      for (auto* t : {&t1, &t2}) {
        t->resize(channels);
        for (int ch = 0; ch < channels; ++ch) {
          const int n = T.i();
          if (n < 0) throw std::runtime_error("data file: bad coefficient table length");
          (*t)[ch].resize(n + 1);
          for (auto& x : (*t)[ch]) x = T.d();
        }
      }
    } else {
      throw std::runtime_error(std::string("Unknown block ") + kind + " in data file.");
    }
    std::string extra;
    if (T.have && (T.cur >> extra)) throw std::runtime_error("data file: unexpected token " + extra);
    T.have = false;
  }
  if (xi.empty()) throw std::runtime_error("data file: no discretization tables");
}

}  // namespace nrgb
