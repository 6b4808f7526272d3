// QS coefficient tables derived from spin coupling, for 1, 2 and 3 channels.
//
// The reference ships these tables as Mathematica output (coefnew/qs/
// qs-<P>ch-*.dat, included by src/sym-QS.cc and src/nrg-recalc-QS.cc).
// Here they are computed from their definition:
//   * a subspace I = (Q, SS) of step N+1 is spanned, for each combination i,
//     by  sum_{m_a, m_s} <S_a m_a; s_i m_s | S M> |site_i m_s> |anc_i m_a>,
//     anc_i = I + In[i] a subspace of step N and site_i a spin multiplet of
//     the added site with fixed electron numbers per channel (three channels
//     have two spin-1/2 multiplets with one electron per channel, told apart
//     by the spin to which channels 0 and 1 couple);
//   * the added site's fermion operators stand to the left of the chain's,
//     so an odd chain operator picks up (-1)^(electrons on the site);
//   * chain operators enter through reduced matrix elements in the
//     Wigner-Eckart normalisation <S1 M1|T^k_q|S2 M2> = <S2 M2; k q|S1 M1> R.
// Every entry is a matrix element in the site's Fock space (4, 16 or 64 states)
// divided by the Clebsch-Gordan coefficient of the Wigner-Eckart theorem.
// The phases of the site multiplets are the reference's conventions.
#pragma once
#include <math.h>

#include <map>
#include <vector>

#include "data.h"

namespace nrgb {

// 1-based combination indices.  kind 0: hopping xi_N <||f^dag||>; 1:
// anomalous hopping kappa_N <||f^dag||>; 2: on-site pairing of the new site,
// 2 delta_N+1 times the identity between two combinations of one ancestor.
struct OffdiagTerm { int i, j, ch; double factor; int kind = 0; };
struct DiagTerm { int i, ch; double number; };
struct RecalcRow { int i1, ip; double factor; };
struct RecalcTable { Invar Ip; int ch; std::vector<RecalcRow> rows; };

// <j1 m1; j2 m2 | J M> (Racah's formula; spins and projections as doubles)
double clebsch_gordan(double j1, double m1, double j2, double m2, double J, double M);

// With spsu2 set: the SPSU2 tables (spin SU(2), charge not conserved; the
// combinations of coefnew/spsu2/spsu2-<P>ch-In2.dat; offdiag also returns
// the anomalous hopping (kind 1) and the on-site pairing (kind 2) terms).
class QSCoupling {
 public:
  explicit QSCoupling(int channels, bool spsu2 = false);
  int combs() const { return (int)combos_.size(); }
  const std::vector<Invar>& In() const { return in_; }
  const std::vector<Invar>& QN() const { return qn_; }
  std::vector<DiagTerm> diag() const;
  // cached per multiplicity / subspace
  const std::vector<OffdiagTerm>& offdiag(int ss);
  const std::vector<RecalcTable>& recalc_f(const Invar& Ip);
  const std::vector<RecalcTable>& doublet(const Invar& I1);
  const std::vector<RecalcTable>& triplet(const Invar& I1);

 private:
  struct Combo {
    std::vector<int> occ;  // electrons per channel on the site
    double s;              // site spin
    Invar In;              // ancestor = I + In
    int label = 0;         // which of equal (occ, s) multiplets
    int twos() const { return (int)lround(2 * s); }
  };
  using Vec = std::vector<double>;
  // |state> = sum over 2 m_a of (site vector) |anc m_a>
  struct State {
    std::map<int, Vec> parts;
    double Sa = 0;
  };
  int P_, dim_;
  bool spsu2_ = false;
  std::vector<Vec> pair_;               // per channel: f^dag_up f^dag_dn + h.c. of the site (SPSU2)
  std::vector<Combo> combos_;
  std::vector<Invar> in_, qn_;
  std::vector<Vec> cd_;                 // creation operators, dim x dim, row-major
  Vec sp_;                              // total S+ of the site
  std::map<std::pair<int, int>, std::map<int, Vec>> mult_;  // (occupations and label, 2s) -> 2M -> state
  std::map<int, std::vector<OffdiagTerm>> off_;
  std::map<Invar, std::vector<RecalcTable>> rf_, dbl_, trp_;

  Vec apply(const Vec& op, const Vec& v) const;
  Vec apply_t(const Vec& op, const Vec& v) const;  // transpose
  std::map<int, Vec> multiplet(const std::vector<int>& occ, double s, double sign) const;
  std::map<int, Vec> coupled_doublet(int label, double sign) const;
  std::pair<int, int> mult_key(const Combo& c) const {
    int key = 0;
    for (int ch = 0; ch < P_; ++ch) key = key * 3 + c.occ[ch];
    return {key * 2 + c.label, c.twos()};
  }
  bool state(int i, double S, double M, State& out) const;
  Invar anc(int i, const Invar& I) const { return {I.first + combos_[i].In.first, I.second + combos_[i].In.second}; }
  int nsite(int i) const;
  double elem(int i, double S1, double M1, int j, double S2, double M2, double rank, double q, const Vec* site_op,
              bool transpose_op, bool odd) const;
  template <class F>
  double reduced(const Invar& I1, const Invar& Ip, double rank, F comp) const;
  std::vector<RecalcRow> chain_op(const Invar& I1, const Invar& Ip, double rank, bool odd) const;
};

}  // namespace nrgb
