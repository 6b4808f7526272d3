// Symmetry plug-in interface of the NRG step (the role of class Symmetry,
// src/symmetry.cc:64-221) and the QS plug-in: charge U(1) x spin SU(2),
// invariant subspaces (Q, SS) with SS = 2S+1 (src/sym-QS.cc).
//
// The host expands these tables into flat task lists (assembly terms, GEMM
// segments) that the device executes; the kernels never see quantum numbers.
//
// The 1-channel QS coefficient tables restate coefnew/qs/qs-1ch-*.dat, each
// Clebsch-Gordan expression simplified to a closed form in SS; the
// 2-channel tables are derived from spin coupling (qs_coupling.h).  Both are
// checked entry by entry against the reference tables by the test suite.
#pragma once
#include <math.h>

#include <stdexcept>
#include <string>
#include <vector>

#include <memory>

#include "data.h"
#include "qs_coupling.h"

namespace nrgb {


class Symmetry {
 public:
  virtual ~Symmetry() = default;
  virtual std::string name() const = 0;
  virtual int combs() const = 0;
  virtual const std::vector<Invar>& In() const = 0;   // ancestor = I + In[i]
  virtual const std::vector<Invar>& QN() const = 0;   // quantum numbers of the added states
  virtual int mult(const Invar& I) const = 0;
  virtual bool allowed(const Invar& I) const = 0;
  virtual bool triangle(const Invar& a, const Invar& b, const Invar& c) const = 0;
  virtual Invar singlet() const = 0;
  virtual Invar doublet() const = 0;
  virtual Invar triplet() const = 0;
  virtual std::vector<OffdiagTerm> offdiag(const Invar& I) const = 0;
  virtual std::vector<DiagTerm> diag() const = 0;
  // <I1||f^dag_ch||Ip> of the new site, for every I1 reachable from Ip
  virtual std::vector<RecalcTable> recalc_f(const Invar& Ip) const = 0;
  // doublet / triplet operator recalculation tables for bra subspace I1
  virtual std::vector<RecalcTable> recalc_doublet(const Invar& I1) const = 0;
  virtual std::vector<RecalcTable> recalc_triplet(const Invar& I1) const = 0;
  virtual double specdens_factor(const Invar& Ip, const Invar& I1) const = 0;
  virtual double dynsusc_factor(const Invar& Ip, const Invar& I1) const = 0;
  // symmetry-specific td columns (names and values from Boltzmann sums)
  virtual std::vector<std::string> td_names() const = 0;
  virtual std::vector<double> td_values(const std::vector<std::pair<Invar, const std::vector<double>*>>& blocks,
                                        double factor, double Z) const = 0;
  // Same from the Boltzmann sums sum_r e^(-factor E_r) of each block.
  virtual std::vector<double> td_values_sums(const std::vector<std::pair<Invar, double>>& zsum, double Z) const = 0;
  // Symmetries with a spin-projection quantum number (a magnetic field is
  // allowed) resolve fermionic spectral functions by spin: SPIN = +1 / -1
  // pairs with SSZ(I1) - SSZ(Ip) = SPIN (isfield, check_SPIN, src/sym-QSZ.cc:26-33,
  // src/nrg.cc:1770-1787).
  virtual bool isfield() const { return false; }
  virtual bool check_spin(const Invar&, const Invar&, int) const { return true; }
  // Whether an operator of kind Iop can connect Ip to I1 (the triangle
  // inequality for SU(2) symmetries; both spin components of a doublet for
  // the spin-projection symmetries).
  virtual bool connects(const Invar& I1, const Invar& Ip, const Invar& Iop) const { return triangle(I1, Ip, Iop); }
  // The quantum numbers of a subspace as the reference prints them
  // (annotated.dat): both numbers, or the spin alone for SPSU2.
  virtual std::string label(const Invar& I) const { return std::to_string(I.first) + " " + std::to_string(I.second); }
  static Invar combine(const Invar& a, const Invar& b) { return {a.first + b.first, a.second + b.second}; }
  static Invar inverse(const Invar& a) { return {-a.first, -a.second}; }
};

class SymmetryQS : public Symmetry {
 public:
  explicit SymmetryQS(int channels) : nch_(channels) {
    if (channels == 2 || channels == 3) {
      cpl_.reset(new QSCoupling(channels));
      in_ = cpl_->In();
      qn_ = cpl_->QN();
      return;
    }
    if (channels != 1) throw std::runtime_error("QS symmetry: this build provides the 1-, 2- and 3-channel tables");
    in_ = {{1, 0}, {0, -1}, {0, 1}, {-1, 0}};
    qn_ = {{-1, 1}, {0, 2}, {0, 2}, {1, 1}};
  }
  std::string name() const override { return "QS"; }
  int combs() const override { return cpl_ ? cpl_->combs() : 4; }
  const std::vector<Invar>& In() const override { return in_; }
  const std::vector<Invar>& QN() const override { return qn_; }
  int mult(const Invar& I) const override { return I.second; }
  bool allowed(const Invar& I) const override { return I.second > 0; }
  static bool su2(int a, int b, int c) {
    return abs(a - b) <= c - 1 && abs(b - c) <= a - 1 && abs(c - a) <= b - 1;
  }
  bool triangle(const Invar& a, const Invar& b, const Invar& c) const override {
    return a.first == b.first + c.first && su2(a.second, b.second, c.second);
  }
  Invar singlet() const override { return {0, 1}; }
  Invar doublet() const override { return {1, 2}; }
  Invar triplet() const override { return {0, 3}; }

  std::vector<OffdiagTerm> offdiag(const Invar& I) const override {
    if (cpl_) return cpl_->offdiag(I.second);
    const double ss = I.second;
    return {{1, 2, 0, 1.0}, {1, 3, 0, 1.0}, {2, 4, 0, -sqrt((ss - 1) / ss)}, {3, 4, 0, sqrt((ss + 1) / ss)}};
  }
  std::vector<DiagTerm> diag() const override {
    if (cpl_) return cpl_->diag();
    return {{1, 0, 0.0}, {2, 0, 1.0}, {3, 0, 1.0}, {4, 0, 2.0}};
  }

  std::vector<RecalcTable> recalc_f(const Invar& Ip) const override {
    if (cpl_) return cpl_->recalc_f(Ip);
    const int qp = Ip.first, ssp = Ip.second;
    std::vector<RecalcTable> t;
    t.push_back({{qp + 1, ssp + 1}, 0, {{2, 1, 1.0}, {4, 3, -sqrt(double(ssp) / (ssp + 1))}}});
    if (ssp > 1) t.push_back({{qp + 1, ssp - 1}, 0, {{3, 1, 1.0}, {4, 2, sqrt(double(ssp) / (ssp - 1))}}});
    return t;
  }
  std::vector<RecalcTable> recalc_doublet(const Invar& I1) const override {
    if (cpl_) return cpl_->doublet(I1);
    const int q1 = I1.first, ss1 = I1.second;
    const double c = sqrt(double(ss1 - 1) * (ss1 + 1)) / ss1;
    return {{{q1 - 1, ss1 + 1}, 0, {{1, 1, 1.0}, {2, 2, -c}, {3, 2, 1.0 / ss1}, {3, 3, -1.0}, {4, 4, 1.0}}},
            {{q1 - 1, ss1 - 1}, 0, {{1, 1, 1.0}, {2, 2, -1.0}, {2, 3, -1.0 / ss1}, {3, 3, -c}, {4, 4, 1.0}}}};
  }
  std::vector<RecalcTable> recalc_triplet(const Invar& I1) const override {
    if (cpl_) return cpl_->triplet(I1);
    const int q1 = I1.first, ss1 = I1.second;
    const double S = (ss1 - 1) / 2.0;
    std::vector<RecalcTable> t;
    if (S > 0) {
      const double t22 = sqrt(1 - 1 / S + 2 / (1 + 2 * S));
      const double t23 = 1 / sqrt((1 + S) * (1 + 2 * S));
      const double t32 = -1 / sqrt(S * (1 + 2 * S));
      const double t33 = sqrt(S * (1 + 2 * S) / (pow(1 + S, 3) * (3 + 2 * S))) * (1 + S) +
                         2 * sqrt(S / (3 + 11 * S + 12 * S * S + 4 * S * S * S));
      t.push_back({{q1, ss1}, 0, {{1, 1, 1.0}, {2, 2, t22}, {2, 3, t23}, {3, 2, t32}, {3, 3, t33}, {4, 4, 1.0}}});
    } else {
      t.push_back({{q1, ss1}, 0, {{1, 1, 1.0}, {4, 4, 1.0}}});
    }
    t.push_back({{q1, ss1 + 2}, 0,
                 {{1, 1, 1.0}, {2, 2, sqrt(1 + 1 / (1 + S) - 2 / (1 + 2 * S))},
                  {3, 2, -1 / sqrt((1 + S) * (1 + 2 * S))}, {3, 3, 1.0}, {4, 4, 1.0}}});
    if (S > 0.5) {
      const double m33 = (sqrt((-1 + 4 * S * S) / (S + S * S)) + sqrt((-1 + 2 * S) / (S + 3 * S * S + 2 * S * S * S))) / 2;
      t.push_back({{q1, ss1 - 2}, 0, {{1, 1, 1.0}, {2, 2, 1.0}, {2, 3, 1 / sqrt(S * (1 + 2 * S))}, {3, 3, m33}, {4, 4, 1.0}}});
    }
    return t;
  }
  double specdens_factor(const Invar& Ip, const Invar& I1) const override {
    const double Sp = (Ip.second - 1) / 2.0;
    return I1.second == Ip.second + 1 ? Sp + 1.0 : Sp;
  }
  double dynsusc_factor(const Invar& Ip, const Invar& I1) const override {
    const int ssp = Ip.second, ss1 = I1.second;
    if (ss1 == ssp + 2) return 1.0 + (ssp - 1) / 3.0;
    if (ss1 == ssp) return ssp / 3.0;
    if (ss1 == ssp - 2) return (-2.0 + ssp) / 3.0;
    throw std::runtime_error("dynsusc_factor: not a triplet pair");
  }
  std::vector<std::string> td_names() const override { return {"<Sz^2>", "<Q>", "<Q^2>"}; }
  std::vector<double> td_values(const std::vector<std::pair<Invar, const std::vector<double>*>>& blocks,
                                double factor, double Z) const override {
    double trSZ = 0, trQ = 0, trQ2 = 0;
    for (const auto& b : blocks) {
      double sumZ = 0;
      for (double x : *b.second) sumZ += exp(-factor * x);
      sumZ *= mult(b.first);
      const double q = b.first.first, ss = b.first.second;
      trQ += sumZ * q;
      trQ2 += sumZ * q * q;
      trSZ += sumZ * (ss * ss - 1) / 12.0;
    }
    return {trSZ / Z, trQ / Z, trQ2 / Z};
  }
  std::vector<double> td_values_sums(const std::vector<std::pair<Invar, double>>& zsum, double Z) const override {
    double trSZ = 0, trQ = 0, trQ2 = 0;
    for (const auto& b : zsum) {
      const double sumZ = b.second * mult(b.first);
      const double q = b.first.first, ss = b.first.second;
      trQ += sumZ * q;
      trQ2 += sumZ * q * q;
      trSZ += sumZ * (ss * ss - 1) / 12.0;
    }
    return {trSZ / Z, trQ / Z, trQ2 / Z};
  }

 private:
  int nch_;
  std::unique_ptr<QSCoupling> cpl_;  // derived tables (2 channels)
  std::vector<Invar> in_, qn_;
};

// SPSU2 plug-in: spin SU(2) without charge conservation (superconducting
// baths), invariant subspaces SS = 2S+1, written (0, SS) (src/sym-SPSU2.cc),
// one channel.  The combinations of a subspace SS add the new site empty
// (ancestor SS), doubly occupied (ancestor SS), singly occupied on an
// ancestor SS-1 and on an ancestor SS+1 (spsu2-1ch-In2.dat, QN.dat).  With
// S = (SS-1)/2 and a = sqrt((SS-1)/SS), b = sqrt((SS+1)/SS):
//  * hopping xi_N sum_s (f^dag_N,s f_N+1,s + h.c.): (1,3) 1, (1,4) 1,
//    (3,2) -a, (4,2) b (spsu2-1ch-offdiag.dat);
//  * anomalous hopping kappa_N (f^dag_N,up f^dag_N+1,dn - f^dag_N,dn
//    f^dag_N+1,up + h.c.): (2,3) 1, (2,4) 1, (3,1) a, (4,1) -b
//    (spsu2-1ch-anomalous.dat);
//  * on-site pairing delta_N+1 (f^dag_N+1,up f^dag_N+1,dn + h.c.): the
//    empty and the doubly occupied combinations, -1/2 times 2 delta
//    (spsu2-1ch-isospinx.dat; ISOSPINX and ANOMALOUS, src/sym-SPSU2.cc:107-113);
//  * electrons of the new site 0, 2, 1, 1 (spsu2-1ch-diag.dat).
// The <f^dag>, doublet and triplet recalculation tables are those of QS with
// the combinations renumbered (QS 1, 2, 3, 4 = SPSU2 1, 3, 4, 2) and the
// charge dropped.  oracle/spsu2_derive.py derives every entry from the
// site's Fock space; the tests check both against the reference's tables.
// Thermodynamics column <Sz^2> (calculate_TD, src/sym-SPSU2.cc:81-94).
class SymmetrySPSU2 : public Symmetry {
 public:
  // One channel: the closed forms below; two and three channels: the tables
  // derived by QSCoupling in its SPSU2 mode (the 16 or 64 combinations of
  // coefnew/spsu2/spsu2-<P>ch-In2.dat), checked against the reference's by
  // the tests.
  explicit SymmetrySPSU2(int channels = 1) {
    if (channels == 2 || channels == 3) {
      cpl_.reset(new QSCoupling(channels, true));
      in_ = cpl_->In();
      qn_ = cpl_->QN();
      return;
    }
    if (channels != 1) throw std::runtime_error("SPSU2 symmetry: this build provides the 1-, 2- and 3-channel tables");
    in_ = {{0, 0}, {0, 0}, {0, -1}, {0, 1}};
    qn_ = {{0, 1}, {0, 1}, {0, 2}, {0, 2}};
  }
  std::string name() const override { return "SPSU2"; }
  std::string label(const Invar& I) const override { return std::to_string(I.second); }
  int combs() const override { return cpl_ ? cpl_->combs() : 4; }
  const std::vector<Invar>& In() const override { return in_; }
  const std::vector<Invar>& QN() const override { return qn_; }
  int mult(const Invar& I) const override { return I.second; }
  bool allowed(const Invar& I) const override { return I.second > 0; }
  bool triangle(const Invar& a, const Invar& b, const Invar& c) const override {
    return SymmetryQS::su2(a.second, b.second, c.second);
  }
  Invar singlet() const override { return {0, 1}; }
  Invar doublet() const override { return {0, 2}; }
  Invar triplet() const override { return {0, 3}; }

  std::vector<OffdiagTerm> offdiag(const Invar& I) const override {
    if (cpl_) return cpl_->offdiag(I.second);
    const double ss = I.second;
    const double a = sqrt((ss - 1) / ss), b = sqrt((ss + 1) / ss);
    return {{1, 3, 0, 1.0, 0}, {1, 4, 0, 1.0, 0}, {3, 2, 0, -a, 0}, {4, 2, 0, b, 0},
            {2, 3, 0, 1.0, 1}, {2, 4, 0, 1.0, 1}, {3, 1, 0, a, 1},  {4, 1, 0, -b, 1},
            {1, 2, 0, -0.5, 2}};
  }
  std::vector<DiagTerm> diag() const override {
    if (cpl_) return cpl_->diag();
    return {{1, 0, 0.0}, {2, 0, 2.0}, {3, 0, 1.0}, {4, 0, 1.0}};
  }

  std::vector<RecalcTable> recalc_f(const Invar& Ip) const override {
    if (cpl_) return cpl_->recalc_f(Ip);
    const int ssp = Ip.second;
    std::vector<RecalcTable> t;
    t.push_back({{0, ssp + 1}, 0, {{2, 4, -sqrt(double(ssp) / (ssp + 1))}, {3, 1, 1.0}}});
    if (ssp > 1) t.push_back({{0, ssp - 1}, 0, {{2, 3, sqrt(double(ssp) / (ssp - 1))}, {4, 1, 1.0}}});
    return t;
  }
  std::vector<RecalcTable> recalc_doublet(const Invar& I1) const override {
    if (cpl_) return cpl_->doublet(I1);
    const int ss1 = I1.second;
    const double c = sqrt(double(ss1 - 1) * (ss1 + 1)) / ss1;
    std::vector<RecalcTable> t;
    t.push_back({{0, ss1 + 1}, 0, {{1, 1, 1.0}, {2, 2, 1.0}, {3, 3, -c}, {4, 3, 1.0 / ss1}, {4, 4, -1.0}}});
    if (ss1 > 1)
      t.push_back({{0, ss1 - 1}, 0, {{1, 1, 1.0}, {2, 2, 1.0}, {3, 3, -1.0}, {3, 4, -1.0 / ss1}, {4, 4, -c}}});
    return t;
  }
  std::vector<RecalcTable> recalc_triplet(const Invar& I1) const override {
    if (cpl_) return cpl_->triplet(I1);
    const int ss1 = I1.second;
    const double S = (ss1 - 1) / 2.0;
    std::vector<RecalcTable> t;
    if (S > 0) {
      const double t33 = sqrt(1 - 1 / S + 2 / (1 + 2 * S));
      const double t34 = 1 / sqrt((1 + S) * (1 + 2 * S));
      const double t43 = -1 / sqrt(S * (1 + 2 * S));
      const double t44 = sqrt(S * (1 + 2 * S) / (pow(1 + S, 3) * (3 + 2 * S))) * (1 + S) +
                         2 * sqrt(S / (3 + 11 * S + 12 * S * S + 4 * S * S * S));
      t.push_back({{0, ss1}, 0, {{1, 1, 1.0}, {2, 2, 1.0}, {3, 3, t33}, {3, 4, t34}, {4, 3, t43}, {4, 4, t44}}});
    }
    t.push_back({{0, ss1 + 2}, 0,
                 {{1, 1, 1.0}, {2, 2, 1.0}, {3, 3, sqrt(1 + 1 / (1 + S) - 2 / (1 + 2 * S))},
                  {4, 3, -1 / sqrt((1 + S) * (1 + 2 * S))}, {4, 4, 1.0}}});
    if (S > 0.5) {
      const double m44 = (sqrt((-1 + 4 * S * S) / (S + S * S)) + sqrt((-1 + 2 * S) / (S + 3 * S * S + 2 * S * S * S))) / 2;
      t.push_back({{0, ss1 - 2}, 0, {{1, 1, 1.0}, {2, 2, 1.0}, {3, 3, 1.0}, {3, 4, 1 / sqrt(S * (1 + 2 * S))}, {4, 4, m44}}});
    }
    return t;
  }
  double specdens_factor(const Invar& Ip, const Invar& I1) const override {
    const double Sp = (Ip.second - 1) / 2.0;
    return I1.second == Ip.second + 1 ? Sp + 1.0 : Sp;
  }
  double dynsusc_factor(const Invar& Ip, const Invar& I1) const override {
    const int ssp = Ip.second, ss1 = I1.second;
    if (ss1 == ssp + 2) return 1.0 + (ssp - 1) / 3.0;
    if (ss1 == ssp) return ssp / 3.0;
    if (ss1 == ssp - 2) return (-2.0 + ssp) / 3.0;
    throw std::runtime_error("dynsusc_factor: not a triplet pair");
  }
  std::vector<std::string> td_names() const override { return {"<Sz^2>"}; }
  std::vector<double> td_values(const std::vector<std::pair<Invar, const std::vector<double>*>>& blocks,
                                double factor, double Z) const override {
    double trSZ = 0;
    for (const auto& b : blocks) {
      double sumZ = 0;
      for (double x : *b.second) sumZ += exp(-factor * x);
      const double ss = b.first.second;
      trSZ += sumZ * mult(b.first) * (ss * ss - 1) / 12.0;
    }
    return {trSZ / Z};
  }
  std::vector<double> td_values_sums(const std::vector<std::pair<Invar, double>>& zsum, double Z) const override {
    double trSZ = 0;
    for (const auto& b : zsum) {
      const double ss = b.first.second;
      trSZ += b.second * mult(b.first) * (ss * ss - 1) / 12.0;
    }
    return {trSZ / Z};
  }

 private:
  std::unique_ptr<QSCoupling> cpl_;  // derived tables (2 channels)
  std::vector<Invar> in_, qn_;
};

// QSZ plug-in: charge U(1) x spin-projection U(1), invariant subspaces
// (Q, SSZ) with SSZ = 2 S_z (src/sym-QSZ.cc), one to three channels.  Every
// state is its own multiplet (mult 1); both spin components of f^dag share
// one list of matrix elements <I1|f^dag_sigma|I2> per channel, I1 = I2 +
// (1, +-1) (the reference's perchannel = 1 for QSZ, src/read-input.cc:67-74).
//
// Without spin multiplets every combination of a subspace is one Fock state
// of the added site (modes 2 ch + spin, spin up first, creation operators
// applied in increasing mode order, phase +1) on an ancestor I - QN(state);
// the tables follow from the site's operators alone:
//  * hopping f^dag_N,ch,s f_N+1,ch,s (+ h.c.) between combinations i < j:
//    the site's f_ch,s takes state j to state i (sign from the modes below)
//    and f^dag_N,ch,s passes the n_i site electrons of i (qsz-<P>ch-offdiag);
//  * <f^dag_ch,s> of the new site between combinations of one ancestor
//    (qsz-<P>ch-spinup*, spindown*);
//  * doublet operators of the chain through the site: rows (i, i) with sign
//    (-1)^n_i (qsz-<P>ch-doubletp, doubletm);
//  * electrons of the new site per channel (qsz-<P>ch-diag).
// The combinations are listed in the reference's order (its In2/QN tables);
// the tests check every table entry against the reference's for 1 to 3
// channels.  Thermodynamics columns <Sz^2>, <Sz>, <Q>, <Q^2> (calculate_TD,
// src/sym-QSZ.cc:73-94).  Doublet operators and their spin-resolved
// spectral functions are provided; triplet operators are not.
class SymmetryQSZ : public Symmetry {
 public:
  explicit SymmetryQSZ(int channels = 1) : nch_(channels) {
    // site Fock states of the combinations (bit 2 ch + s: channel ch, spin s = 0 up, 1 down)
    static const int COMB_1CH[] = {0x0, 0x2, 0x1, 0x3};
    static const int COMB_2CH[] = {0x0, 0x8, 0x2, 0x4, 0x1, 0xA, 0xC, 0x6, 0x9, 0x3, 0x5, 0xE, 0xB, 0xD, 0x7, 0xF};
    static const int COMB_3CH[] = {
        0x00, 0x20, 0x08, 0x02, 0x10, 0x04, 0x01, 0x28, 0x22, 0x0A, 0x30, 0x18, 0x24, 0x0C, 0x12, 0x06,
        0x21, 0x09, 0x03, 0x14, 0x11, 0x05, 0x2A, 0x38, 0x2C, 0x32, 0x1A, 0x26, 0x0E, 0x29, 0x23, 0x0B,
        0x34, 0x1C, 0x16, 0x31, 0x19, 0x25, 0x0D, 0x13, 0x07, 0x15, 0x3A, 0x2E, 0x2B, 0x3C, 0x36, 0x1E,
        0x39, 0x2D, 0x33, 0x1B, 0x27, 0x0F, 0x35, 0x1D, 0x17, 0x3E, 0x3B, 0x2F, 0x3D, 0x37, 0x1F, 0x3F};
    if (channels < 1 || channels > 3) throw std::runtime_error("QSZ symmetry: this build provides 1 to 3 channels");
    const int* cb = channels == 1 ? COMB_1CH : channels == 2 ? COMB_2CH : COMB_3CH;
    const int n = 1 << (2 * channels);
    for (int i = 0; i < n; ++i) {
      bits_.push_back(cb[i]);
      int ne = 0, sz = 0;
      for (int m = 0; m < 2 * channels; ++m)
        if ((cb[i] >> m) & 1) {
          ++ne;
          sz += (m & 1) ? -1 : 1;
        }
      qn_.push_back({ne - channels, sz});
      in_.push_back({channels - ne, -sz});
    }
    // hopping terms (they do not depend on the subspace)
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        for (int ch = 0; ch < channels; ++ch) {
          double v = 0.0;
          for (int sp = 0; sp < 2; ++sp) {
            int b = 0;
            const int sg = annihilate(bits_[j], 2 * ch + sp, b);
            if (sg && b == bits_[i]) v += sg * ((popc(bits_[i]) & 1) ? -1.0 : 1.0);
          }
          if (v != 0.0) off_.push_back({i + 1, j + 1, ch, v});
        }
  }
  std::string name() const override { return "QSZ"; }
  int combs() const override { return (int)bits_.size(); }
  const std::vector<Invar>& In() const override { return in_; }
  const std::vector<Invar>& QN() const override { return qn_; }
  int mult(const Invar&) const override { return 1; }
  bool allowed(const Invar&) const override { return true; }
  bool triangle(const Invar& a, const Invar& b, const Invar& c) const override {
    return a.first == b.first + c.first && a.second == b.second + c.second;
  }
  Invar singlet() const override { return {0, 0}; }
  Invar doublet() const override { return {1, 1}; }
  Invar triplet() const override { return {0, 2}; }
  std::vector<OffdiagTerm> offdiag(const Invar&) const override { return off_; }
  std::vector<DiagTerm> diag() const override {
    std::vector<DiagTerm> out;
    for (int ch = 0; ch < nch_; ++ch)
      for (int i = 0; i < combs(); ++i)
        out.push_back({i + 1, ch, (double)(((bits_[i] >> (2 * ch)) & 1) + ((bits_[i] >> (2 * ch + 1)) & 1))});
    return out;
  }
  std::vector<RecalcTable> recalc_f(const Invar& Ip) const override {
    std::vector<RecalcTable> out;
    for (int sp = 0; sp < 2; ++sp)  // up: I1 = Ip + (1, 1); down: Ip + (1, -1)
      for (int ch = 0; ch < nch_; ++ch) {
        const Invar I1{Ip.first + 1, Ip.second + (sp ? -1 : 1)};
        RecalcTable t{I1, ch, {}};
        for (int i1 = 0; i1 < combs(); ++i1)
          for (int ip = 0; ip < combs(); ++ip) {
            if (combine(in_[i1], I1) != combine(in_[ip], Ip)) continue;
            int b = 0;
            const int sg = create(bits_[ip], 2 * ch + sp, b);
            if (sg && b == bits_[i1]) t.rows.push_back({i1 + 1, ip + 1, (double)sg});
          }
        out.push_back(t);
      }
    return out;
  }
  // Doublet operators (d^dag_s of the impurity) recalculated through the new
  // site: d^dag passes the n_i electrons of the site, rows (i, i) with sign
  // (-1)^n_i, for the spin-up component (Ip = I1 - (1, 1)) and the spin-down
  // one (Ip = I1 - (1, -1)) (qsz-<P>ch-doubletp.dat, qsz-<P>ch-doubletm.dat).
  std::vector<RecalcTable> recalc_doublet(const Invar& I1) const override {
    const int q1 = I1.first, z1 = I1.second;
    std::vector<RecalcRow> rows;
    for (int i = 0; i < combs(); ++i) rows.push_back({i + 1, i + 1, (popc(bits_[i]) & 1) ? -1.0 : 1.0});
    return {{{q1 - 1, z1 - 1}, 0, rows}, {{q1 - 1, z1 + 1}, 0, rows}};
  }
  std::vector<RecalcTable> recalc_triplet(const Invar&) const override {
    throw std::runtime_error("QSZ: triplet operators are not built");
  }
  bool isfield() const override { return true; }
  bool check_spin(const Invar& I1, const Invar& Ip, int spin) const override {
    return I1.second - Ip.second == spin;
  }
  bool connects(const Invar& I1, const Invar& Ip, const Invar& Iop) const override {
    if (Iop == doublet()) return I1.first == Ip.first + 1 && abs(I1.second - Ip.second) == 1;
    return triangle(I1, Ip, Iop);
  }
  // every state is its own multiplet: no degeneracy factor (the default of
  // Symmetry::specdens_factor, src/symmetry.cc:170-173)
  double specdens_factor(const Invar&, const Invar&) const override { return 1.0; }
  double dynsusc_factor(const Invar&, const Invar&) const override {
    throw std::runtime_error("QSZ: spectral functions are not built");
  }
  std::vector<std::string> td_names() const override { return {"<Sz^2>", "<Sz>", "<Q>", "<Q^2>"}; }
  std::vector<double> td_values(const std::vector<std::pair<Invar, const std::vector<double>*>>& blocks,
                                double factor, double Z) const override {
    std::vector<std::pair<Invar, double>> zs;
    for (const auto& b : blocks) {
      double sumZ = 0;
      for (double x : *b.second) sumZ += exp(-factor * x);
      zs.push_back({b.first, sumZ});
    }
    return td_values_sums(zs, Z);
  }
  std::vector<double> td_values_sums(const std::vector<std::pair<Invar, double>>& zsum, double Z) const override {
    double trSZ = 0, trSZ2 = 0, trQ = 0, trQ2 = 0;
    for (const auto& b : zsum) {
      const double sz = 0.5 * b.first.second, q = b.first.first;
      trSZ += b.second * sz;
      trSZ2 += b.second * sz * sz;
      trQ += b.second * q;
      trQ2 += b.second * q * q;
    }
    return {trSZ2 / Z, trSZ / Z, trQ / Z, trQ2 / Z};
  }

 private:
  static int popc(int b) { return __builtin_popcount((unsigned)b); }
  // sign of the fermion operator on Fock state b (modes below m counted), 0 if it vanishes
  static int create(int b, int m, int& out) {
    if ((b >> m) & 1) return 0;
    out = b | (1 << m);
    return (popc(b & ((1 << m) - 1)) & 1) ? -1 : 1;
  }
  static int annihilate(int b, int m, int& out) {
    if (!((b >> m) & 1)) return 0;
    out = b & ~(1 << m);
    return (popc(b & ((1 << m) - 1)) & 1) ? -1 : 1;
  }
  int nch_;
  std::vector<int> bits_;
  std::vector<Invar> in_, qn_;
  std::vector<OffdiagTerm> off_;
};

}  // namespace nrgb
