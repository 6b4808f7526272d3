// QS coefficient tables derived from spin coupling (see qs_coupling.h).
#include "qs_coupling.h"

#include <math.h>

#include <algorithm>
#include <stdexcept>

namespace nrgb {

namespace {

// Combinations of a new subspace, in the reference's order (the In2, QN and
// diag tables of coefnew/qs/qs-<P>ch-*.dat): electrons per channel on the
// added site, site spin, In = ancestor - subspace.
struct ComboDef {
  int occ[3];
  double s;
  int dq, dss;
  int label = 0;
};
const ComboDef COMBOS_1CH[] = {{{0, 0}, 0.0, 1, 0}, {{1, 0}, 0.5, 0, -1}, {{1, 0}, 0.5, 0, 1}, {{2, 0}, 0.0, -1, 0}};
const ComboDef COMBOS_2CH[] = {{{0, 0}, 0.0, 2, 0},   {{0, 1}, 0.5, 1, -1},  {{0, 1}, 0.5, 1, 1},
                               {{1, 0}, 0.5, 1, -1},  {{1, 0}, 0.5, 1, 1},   {{0, 2}, 0.0, 0, 0},
                               {{1, 1}, 0.0, 0, 0},   {{2, 0}, 0.0, 0, 0},   {{1, 1}, 1.0, 0, -2},
                               {{1, 1}, 1.0, 0, 0},   {{1, 1}, 1.0, 0, 2},   {{1, 2}, 0.5, -1, -1},
                               {{1, 2}, 0.5, -1, 1},  {{2, 1}, 0.5, -1, -1}, {{2, 1}, 0.5, -1, 1},
                               {{2, 2}, 0.0, -2, 0}};

// Three channels (coefnew/qs/qs-3ch-In2.dat, QN, diag); label 1 marks the
// second spin-1/2 multiplet with one electron per channel.
const ComboDef COMBOS_3CH[] = {
    {{0, 0, 0}, 0.0, 3, 0}, {{0, 0, 1}, 0.5, 2, -1}, {{0, 0, 1}, 0.5, 2, 1}, {{0, 1, 0}, 0.5, 2, -1},
    {{0, 1, 0}, 0.5, 2, 1}, {{1, 0, 0}, 0.5, 2, -1}, {{1, 0, 0}, 0.5, 2, 1}, {{0, 0, 2}, 0.0, 1, 0},
    {{0, 1, 1}, 0.0, 1, 0}, {{1, 0, 1}, 0.0, 1, 0}, {{0, 2, 0}, 0.0, 1, 0}, {{1, 1, 0}, 0.0, 1, 0},
    {{2, 0, 0}, 0.0, 1, 0}, {{0, 1, 1}, 1.0, 1, -2}, {{0, 1, 1}, 1.0, 1, 0}, {{0, 1, 1}, 1.0, 1, 2},
    {{1, 0, 1}, 1.0, 1, -2}, {{1, 0, 1}, 1.0, 1, 0}, {{1, 0, 1}, 1.0, 1, 2}, {{1, 1, 0}, 1.0, 1, -2},
    {{1, 1, 0}, 1.0, 1, 0}, {{1, 1, 0}, 1.0, 1, 2}, {{0, 1, 2}, 0.5, 0, -1}, {{0, 1, 2}, 0.5, 0, 1},
    {{1, 0, 2}, 0.5, 0, -1}, {{1, 0, 2}, 0.5, 0, 1}, {{0, 2, 1}, 0.5, 0, -1}, {{0, 2, 1}, 0.5, 0, 1},
    {{1, 1, 1}, 0.5, 0, -1}, {{1, 1, 1}, 0.5, 0, 1}, {{2, 0, 1}, 0.5, 0, -1}, {{2, 0, 1}, 0.5, 0, 1},
    {{1, 1, 1}, 0.5, 0, -1, 1}, {{1, 1, 1}, 0.5, 0, 1, 1}, {{1, 2, 0}, 0.5, 0, -1}, {{1, 2, 0}, 0.5, 0, 1},
    {{2, 1, 0}, 0.5, 0, -1}, {{2, 1, 0}, 0.5, 0, 1}, {{1, 1, 1}, 1.5, 0, -3}, {{1, 1, 1}, 1.5, 0, -1},
    {{1, 1, 1}, 1.5, 0, 1}, {{1, 1, 1}, 1.5, 0, 3}, {{0, 2, 2}, 0.0, -1, 0}, {{1, 1, 2}, 0.0, -1, 0},
    {{2, 0, 2}, 0.0, -1, 0}, {{1, 2, 1}, 0.0, -1, 0}, {{2, 1, 1}, 0.0, -1, 0}, {{2, 2, 0}, 0.0, -1, 0},
    {{1, 1, 2}, 1.0, -1, -2}, {{1, 1, 2}, 1.0, -1, 0}, {{1, 1, 2}, 1.0, -1, 2}, {{1, 2, 1}, 1.0, -1, -2},
    {{1, 2, 1}, 1.0, -1, 0}, {{1, 2, 1}, 1.0, -1, 2}, {{2, 1, 1}, 1.0, -1, -2}, {{2, 1, 1}, 1.0, -1, 0},
    {{2, 1, 1}, 1.0, -1, 2}, {{1, 2, 2}, 0.5, -2, -1}, {{1, 2, 2}, 0.5, -2, 1}, {{2, 1, 2}, 0.5, -2, -1},
    {{2, 1, 2}, 0.5, -2, 1}, {{2, 2, 1}, 0.5, -2, -1}, {{2, 2, 1}, 0.5, -2, 1}, {{2, 2, 2}, 0.0, -3, 0},
};

// Three-channel site multiplets with the opposite phase: electrons per
// channel, 2s, label.
struct SignDef {
  int occ[3];
  int twos, label;
};
const SignDef NEGATIVE_3CH[] = {
    {{0, 0, 2}, 0, 0}, {{0, 1, 1}, 2, 0}, {{0, 1, 2}, 1, 0}, {{0, 2, 0}, 0, 0},
    {{0, 2, 1}, 1, 0}, {{1, 0, 1}, 2, 0}, {{1, 0, 2}, 1, 0}, {{1, 1, 0}, 2, 0},
    {{1, 1, 1}, 1, 0}, {{1, 1, 1}, 1, 1}, {{1, 1, 1}, 3, 0}, {{1, 1, 2}, 0, 0},
    {{1, 2, 0}, 1, 0}, {{1, 2, 1}, 0, 0}, {{2, 0, 0}, 0, 0}, {{2, 0, 1}, 1, 0},
    {{2, 1, 0}, 1, 0}, {{2, 1, 1}, 0, 0}, {{2, 2, 2}, 0, 0},
};

// The same for SPSU2 (no charge: every In is (0, dss)), in the order of
// coefnew/spsu2/spsu2-<P>ch-In2.dat: site singlets, doublets, the triplet.
const ComboDef SPSU2_1CH[] = {{{0, 0}, 0.0, 0, 0}, {{2, 0}, 0.0, 0, 0}, {{1, 0}, 0.5, 0, -1}, {{1, 0}, 0.5, 0, 1}};
const ComboDef SPSU2_2CH[] = {{{0, 0}, 0.0, 0, 0},  {{0, 2}, 0.0, 0, 0},  {{1, 1}, 0.0, 0, 0},  {{2, 0}, 0.0, 0, 0},
                              {{2, 2}, 0.0, 0, 0},  {{0, 1}, 0.5, 0, -1}, {{0, 1}, 0.5, 0, 1},  {{1, 0}, 0.5, 0, -1},
                              {{1, 0}, 0.5, 0, 1},  {{1, 2}, 0.5, 0, -1}, {{1, 2}, 0.5, 0, 1},  {{2, 1}, 0.5, 0, -1},
                              {{2, 1}, 0.5, 0, 1},  {{1, 1}, 1.0, 0, -2}, {{1, 1}, 1.0, 0, 0},  {{1, 1}, 1.0, 0, 2}};

// Three channels: site singlets, doublets, quartet in the order of
// coefnew/spsu2/spsu2-3ch-In2.dat, QN and diag; label 1 marks the second
// spin-1/2 multiplet with one electron per channel.
const ComboDef SPSU2_3CH[] = {
    {{0, 0, 0}, 0.0, 0, 0}, {{0, 0, 2}, 0.0, 0, 0}, {{0, 1, 1}, 0.0, 0, 0}, {{1, 0, 1}, 0.0, 0, 0},
    {{0, 2, 0}, 0.0, 0, 0}, {{1, 1, 0}, 0.0, 0, 0}, {{2, 0, 0}, 0.0, 0, 0}, {{0, 2, 2}, 0.0, 0, 0},
    {{1, 1, 2}, 0.0, 0, 0}, {{2, 0, 2}, 0.0, 0, 0}, {{1, 2, 1}, 0.0, 0, 0}, {{2, 1, 1}, 0.0, 0, 0},
    {{2, 2, 0}, 0.0, 0, 0}, {{2, 2, 2}, 0.0, 0, 0}, {{0, 0, 1}, 0.5, 0, -1}, {{0, 0, 1}, 0.5, 0, 1},
    {{0, 1, 0}, 0.5, 0, -1}, {{0, 1, 0}, 0.5, 0, 1}, {{1, 0, 0}, 0.5, 0, -1}, {{1, 0, 0}, 0.5, 0, 1},
    {{0, 1, 2}, 0.5, 0, -1}, {{0, 1, 2}, 0.5, 0, 1}, {{1, 0, 2}, 0.5, 0, -1}, {{1, 0, 2}, 0.5, 0, 1},
    {{0, 2, 1}, 0.5, 0, -1}, {{0, 2, 1}, 0.5, 0, 1}, {{1, 1, 1}, 0.5, 0, -1}, {{1, 1, 1}, 0.5, 0, 1},
    {{2, 0, 1}, 0.5, 0, -1}, {{2, 0, 1}, 0.5, 0, 1}, {{1, 1, 1}, 0.5, 0, -1, 1}, {{1, 1, 1}, 0.5, 0, 1, 1},
    {{1, 2, 0}, 0.5, 0, -1}, {{1, 2, 0}, 0.5, 0, 1}, {{2, 1, 0}, 0.5, 0, -1}, {{2, 1, 0}, 0.5, 0, 1},
    {{1, 2, 2}, 0.5, 0, -1}, {{1, 2, 2}, 0.5, 0, 1}, {{2, 1, 2}, 0.5, 0, -1}, {{2, 1, 2}, 0.5, 0, 1},
    {{2, 2, 1}, 0.5, 0, -1}, {{2, 2, 1}, 0.5, 0, 1}, {{0, 1, 1}, 1.0, 0, -2}, {{0, 1, 1}, 1.0, 0, 0},
    {{0, 1, 1}, 1.0, 0, 2}, {{1, 0, 1}, 1.0, 0, -2}, {{1, 0, 1}, 1.0, 0, 0}, {{1, 0, 1}, 1.0, 0, 2},
    {{1, 1, 0}, 1.0, 0, -2}, {{1, 1, 0}, 1.0, 0, 0}, {{1, 1, 0}, 1.0, 0, 2}, {{1, 1, 2}, 1.0, 0, -2},
    {{1, 1, 2}, 1.0, 0, 0}, {{1, 1, 2}, 1.0, 0, 2}, {{1, 2, 1}, 1.0, 0, -2}, {{1, 2, 1}, 1.0, 0, 0},
    {{1, 2, 1}, 1.0, 0, 2}, {{2, 1, 1}, 1.0, 0, -2}, {{2, 1, 1}, 1.0, 0, 0}, {{2, 1, 1}, 1.0, 0, 2},
    {{1, 1, 1}, 1.5, 0, -3}, {{1, 1, 1}, 1.5, 0, -1}, {{1, 1, 1}, 1.5, 0, 1}, {{1, 1, 1}, 1.5, 0, 3},
};

// Phase of each site multiplet relative to the highest-weight state whose
// first nonzero amplitude (bit k = mode k = 2*channel + spin, up first) is
// positive: the reference's conventions.
double site_sign(int P, const std::vector<int>& occ, double s, int label) {
  const int twos = (int)lround(2 * s);
  if (P == 1) return (occ[0] == 2) ? -1.0 : 1.0;
  if (P == 3) {
    for (const SignDef& d : NEGATIVE_3CH)
      if (d.occ[0] == occ[0] && d.occ[1] == occ[1] && d.occ[2] == occ[2] && d.twos == twos && d.label == label)
        return -1.0;
    return 1.0;
  }
  const int a = occ[0], b = occ[1];
  if ((a == 2 && b == 0) || (a == 0 && b == 2)) return -1.0;
  if (a == 1 && b == 1 && twos == 2) return -1.0;
  if ((a == 1 && b == 2) || (a == 2 && b == 1)) return -1.0;
  return 1.0;
}

double lfact(double x) { return lgamma((double)lround(x) + 1.0); }

int popcount(unsigned x) { return __builtin_popcount(x); }

}  // namespace

double clebsch_gordan(double j1, double m1, double j2, double m2, double J, double M) {
  if (fabs(m1 + m2 - M) > 1e-9 || J < fabs(j1 - j2) - 1e-9 || J > j1 + j2 + 1e-9) return 0.0;
  if (fabs(m1) > j1 + 1e-9 || fabs(m2) > j2 + 1e-9 || fabs(M) > J + 1e-9) return 0.0;
  const double pre = 0.5 * (log(2 * J + 1) + lfact(J + j1 - j2) + lfact(J - j1 + j2) + lfact(j1 + j2 - J) -
                            lfact(j1 + j2 + J + 1) + lfact(J + M) + lfact(J - M) + lfact(j1 - m1) + lfact(j1 + m1) +
                            lfact(j2 - m2) + lfact(j2 + m2));
  const long kmin = std::max(0L, std::max(lround(j2 - J - m1), lround(j1 - J + m2)));
  const long kmax = std::min(lround(j1 + j2 - J), std::min(lround(j1 - m1), lround(j2 + m2)));
  double s = 0.0;
  for (long k = kmin; k <= kmax; ++k) {
    const double den = lfact(k) + lfact(j1 + j2 - J - k) + lfact(j1 - m1 - k) + lfact(j2 + m2 - k) +
                       lfact(J - j2 + m1 + k) + lfact(J - j1 - m2 + k);
    s += ((k & 1) ? -1.0 : 1.0) * exp(pre - den);
  }
  return s;
}

QSCoupling::QSCoupling(int channels, bool spsu2) : P_(channels), spsu2_(spsu2) {
  if (channels < 1 || channels > 3)
    throw std::runtime_error(spsu2 ? "SPSU2 symmetry: tables for 1, 2 and 3 channels"
                                   : "QS symmetry: tables for 1, 2 and 3 channels");
  dim_ = 1 << (2 * P_);
  const ComboDef* defs = spsu2 ? (P_ == 1 ? SPSU2_1CH : P_ == 2 ? SPSU2_2CH : SPSU2_3CH)
                               : (P_ == 1 ? COMBOS_1CH : P_ == 2 ? COMBOS_2CH : COMBOS_3CH);
  const int n = 1 << (2 * P_);
  for (int i = 0; i < n; ++i) {
    Combo c;
    c.occ.assign(defs[i].occ, defs[i].occ + P_);
    c.s = defs[i].s;
    c.label = defs[i].label;
    c.In = {defs[i].dq, defs[i].dss};
    combos_.push_back(c);
    in_.push_back(c.In);
    int ne = 0;
    for (int x : c.occ) ne += x;
    qn_.push_back({spsu2 ? 0 : ne - P_, (int)lround(2 * c.s) + 1});
  }
  // creation operators (Jordan-Wigner order of the site's 2P modes)
  const int nm = 2 * P_;
  for (int k = 0; k < nm; ++k) {
    Vec M((size_t)dim_ * dim_, 0.0);
    for (int b = 0; b < dim_; ++b)
      if (!((b >> k) & 1)) M[(size_t)(b | (1 << k)) * dim_ + b] = (popcount(b & ((1u << k) - 1)) & 1) ? -1.0 : 1.0;
    cd_.push_back(M);
  }
  // S+ = sum_ch c^dag_{ch up} c_{ch dn}
  sp_.assign((size_t)dim_ * dim_, 0.0);
  for (int ch = 0; ch < P_; ++ch) {
    const Vec& up = cd_[2 * ch];
    const Vec& dn = cd_[2 * ch + 1];
    for (int r = 0; r < dim_; ++r)
      for (int c = 0; c < dim_; ++c) {
        double t = 0.0;
        for (int k = 0; k < dim_; ++k) t += up[(size_t)r * dim_ + k] * dn[(size_t)c * dim_ + k];  // up * dn^T
        sp_[(size_t)r * dim_ + c] += t;
      }
  }
  for (const Combo& c : combos_) {
    const std::pair<int, int> k2 = mult_key(c);
    if (mult_.count(k2)) continue;
    const double sign = site_sign(P_, c.occ, c.s, c.label);
    if (P_ == 3 && c.occ == std::vector<int>{1, 1, 1} && c.twos() == 1)
      mult_[k2] = coupled_doublet(c.label, sign);
    else
      mult_[k2] = multiplet(c.occ, c.s, sign);
  }
  // the site's pairing operator f^dag_up f^dag_dn + h.c. per channel (SPSU2)
  if (spsu2)
    for (int ch = 0; ch < P_; ++ch) {
      const Vec& a = cd_[2 * ch];
      const Vec& b = cd_[2 * ch + 1];
      Vec pr((size_t)dim_ * dim_, 0.0);
      for (int r = 0; r < dim_; ++r)
        for (int k = 0; k < dim_; ++k) {
          const double x = a[(size_t)r * dim_ + k];
          if (x == 0.0) continue;
          for (int c2 = 0; c2 < dim_; ++c2) pr[(size_t)r * dim_ + c2] += x * b[(size_t)k * dim_ + c2];
        }
      Vec sym(pr);
      for (int r = 0; r < dim_; ++r)
        for (int c2 = 0; c2 < dim_; ++c2) sym[(size_t)r * dim_ + c2] += pr[(size_t)c2 * dim_ + r];
      pair_.push_back(sym);
    }
}

QSCoupling::Vec QSCoupling::apply(const Vec& op, const Vec& v) const {
  Vec w(dim_, 0.0);
  for (int r = 0; r < dim_; ++r) {
    double s = 0.0;
    for (int c = 0; c < dim_; ++c) s += op[(size_t)r * dim_ + c] * v[c];
    w[r] = s;
  }
  return w;
}

QSCoupling::Vec QSCoupling::apply_t(const Vec& op, const Vec& v) const {
  Vec w(dim_, 0.0);
  for (int r = 0; r < dim_; ++r)
    for (int c = 0; c < dim_; ++c) w[c] += op[(size_t)r * dim_ + c] * v[r];
  return w;
}

int QSCoupling::nsite(int i) const {
  int n = 0;
  for (int x : combos_[i].occ) n += x;
  return n;
}

// Spin-s multiplet with the given electrons per channel: the highest-weight
// state (annihilated by S+ within the S_z = s states of that occupation),
// then S- down to M = -s.
std::map<int, QSCoupling::Vec> QSCoupling::multiplet(const std::vector<int>& occ, double s, double sign) const {
  auto sz2 = [&](int b) {
    int t = 0;
    for (int ch = 0; ch < P_; ++ch) t += ((b >> (2 * ch)) & 1) - ((b >> (2 * ch + 1)) & 1);
    return t;
  };
  auto occ_ok = [&](int b) {
    for (int ch = 0; ch < P_; ++ch)
      if (popcount((b >> (2 * ch)) & 3) != occ[ch]) return false;
    return true;
  };
  const int twos = (int)lround(2 * s);
  std::vector<int> idx;
  for (int b = 0; b < dim_; ++b)
    if (occ_ok(b) && sz2(b) == twos) idx.push_back(b);
  const Vec& Sp = sp_;
  // null space of the columns idx of S+: orthonormal basis of the row space
  // (restricted to idx), then the first unit vector with a residual
  const int m = (int)idx.size();
  std::vector<Vec> rows;
  for (int r = 0; r < dim_; ++r) {
    Vec v(m);
    for (int t = 0; t < m; ++t) v[t] = Sp[(size_t)r * dim_ + idx[t]];
    for (const Vec& u : rows) {
      double d = 0;
      for (int t = 0; t < m; ++t) d += u[t] * v[t];
      for (int t = 0; t < m; ++t) v[t] -= d * u[t];
    }
    double nv = 0;
    for (double x : v) nv += x * x;
    if (nv > 1e-18) {
      for (double& x : v) x /= sqrt(nv);
      rows.push_back(v);
    }
  }
  if ((int)rows.size() != m - 1) throw std::runtime_error("QS coupling: site multiplet is not unique");
  Vec hw(m, 0.0);
  for (int e = 0; e < m; ++e) {
    Vec v(m, 0.0);
    v[e] = 1.0;
    for (const Vec& u : rows) {
      const double d = u[e];
      for (int t = 0; t < m; ++t) v[t] -= d * u[t];
    }
    double nv = 0;
    for (double x : v) nv += x * x;
    if (nv > 1e-12) {
      for (int t = 0; t < m; ++t) hw[t] = v[t] / sqrt(nv);
      break;
    }
  }
  Vec st(dim_, 0.0);
  for (int t = 0; t < m; ++t) st[idx[t]] = hw[t];
  double first = 0;
  for (double x : st)
    if (fabs(x) > 1e-9) {
      first = x;
      break;
    }
  for (double& x : st) x *= (first > 0 ? 1.0 : -1.0) * sign;
  std::map<int, Vec> out;
  out[twos] = st;
  double M = s;
  while (M > -s + 1e-9) {
    Vec w = apply_t(Sp, st);  // S- = (S+)^T
    const double nrm = sqrt((s + M) * (s - M + 1));
    for (double& x : w) x /= nrm;
    M -= 1;
    out[(int)lround(2 * M)] = w;
    st = w;
  }
  return out;
}

// The three-channel spin-1/2 multiplet with one electron per channel whose
// channels 0 and 1 couple to spin s01 = label (0 or 1):
//   |1/2 1/2> = sum <s01 m01; 1/2 mc|1/2 1/2> c^dag_{2,mc} |s01 m01>,
//   |s01 m01> = sum <1/2 ma; 1/2 mb|s01 m01> c^dag_{0,ma} c^dag_{1,mb} |0>,
// normalised and multiplied by `sign`; then S- for M = -1/2.
std::map<int, QSCoupling::Vec> QSCoupling::coupled_doublet(int label, double sign) const {
  const double s01 = label;
  Vec vac(dim_, 0.0);
  vac[0] = 1.0;
  auto cdag = [&](int ch, double m, const Vec& v) { return apply(cd_[2 * ch + (m > 0 ? 0 : 1)], v); };
  Vec hw(dim_, 0.0);
  for (double m01 = -s01; m01 <= s01 + 1e-9; m01 += 1.0) {
    Vec pair(dim_, 0.0);
    for (double ma : {0.5, -0.5}) {
      const double g = clebsch_gordan(0.5, ma, 0.5, m01 - ma, s01, m01);
      if (g == 0.0) continue;
      const Vec v = cdag(0, ma, cdag(1, m01 - ma, vac));
      for (int t = 0; t < dim_; ++t) pair[t] += g * v[t];
    }
    const double g = clebsch_gordan(s01, m01, 0.5, 0.5 - m01, 0.5, 0.5);
    if (g == 0.0) continue;
    const Vec v = cdag(2, 0.5 - m01, pair);
    for (int t = 0; t < dim_; ++t) hw[t] += g * v[t];
  }
  double nrm = 0.0;
  for (double x : hw) nrm += x * x;
  for (double& x : hw) x *= sign / sqrt(nrm);
  std::map<int, Vec> out;
  out[1] = hw;
  out[-1] = apply_t(sp_, hw);  // S- |1/2 1/2> = |1/2 -1/2>
  return out;
}

bool QSCoupling::state(int i, double S, double M, State& out) const {
  const Combo& c = combos_[i];
  const double Sa = S + c.In.second / 2.0;
  if (Sa < -1e-9 || S < fabs(Sa - c.s) - 1e-9 || S > Sa + c.s + 1e-9) return false;
  const auto& ms = mult_.at(mult_key(c));
  out.parts.clear();
  out.Sa = Sa;
  for (const auto& kv : ms) {
    const double m_s = kv.first / 2.0;
    const double ma = M - m_s;
    if (fabs(ma) > Sa + 1e-9) continue;
    const double g = clebsch_gordan(Sa, ma, c.s, m_s, S, M);
    if (g == 0.0) continue;
    Vec& p = out.parts[(int)lround(2 * ma)];
    if (p.empty()) p.assign(dim_, 0.0);
    for (int t = 0; t < dim_; ++t) p[t] += g * kv.second[t];
  }
  return true;
}

double QSCoupling::elem(int i, double S1, double M1, int j, double S2, double M2, double rank, double q,
                        const Vec* site_op, bool transpose_op, bool odd) const {
  State a, b;
  if (!state(i, S1, M1, a) || !state(j, S2, M2, b)) return 0.0;
  double tot = 0.0;
  for (const auto& x : a.parts) {
    for (const auto& y : b.parts) {
      double ae;
      if (rank < 0) {
        if (x.first != y.first || fabs(a.Sa - b.Sa) > 1e-9) continue;
        ae = 1.0;
      } else {
        ae = clebsch_gordan(b.Sa, y.first / 2.0, rank, q, a.Sa, x.first / 2.0);
        if (ae == 0.0) continue;
      }
      const Vec w = site_op ? (transpose_op ? apply_t(*site_op, y.second) : apply(*site_op, y.second)) : y.second;
      double d = 0.0;
      for (int t = 0; t < dim_; ++t) d += x.second[t] * w[t];
      tot += ae * d * ((odd && (nsite(i) & 1)) ? -1.0 : 1.0);
    }
  }
  return tot;
}

template <class F>
double QSCoupling::reduced(const Invar& I1, const Invar& Ip, double rank, F comp) const {
  const double S1 = (I1.second - 1) / 2.0, Sp = (Ip.second - 1) / 2.0;
  for (int q2 = (int)lround(-2 * rank); q2 <= (int)lround(2 * rank); q2 += 2) {
    const double q = q2 / 2.0, M2 = S1 - q;
    if (fabs(M2) > Sp + 1e-9) continue;
    const double g = clebsch_gordan(Sp, M2, rank, q, S1, S1);
    if (fabs(g) > 1e-12) return comp(q, S1, Sp, M2) / g;
  }
  return 0.0;
}

std::vector<DiagTerm> QSCoupling::diag() const {
  std::vector<DiagTerm> out;
  for (int ch = 0; ch < P_; ++ch)
    for (int i = 0; i < combs(); ++i) out.push_back({i + 1, ch, (double)combos_[i].occ[ch]});
  return out;
}

const std::vector<OffdiagTerm>& QSCoupling::offdiag(int ss) {
  auto it = off_.find(ss);
  if (it != off_.end()) return it->second;
  const double S = (ss - 1) / 2.0;
  std::vector<OffdiagTerm> out;
  const int n = combs();
  // QS: the combinations are ordered by the site's electrons, so the hopping
  // connects i < j only; SPSU2: every ordered pair, and the anomalous
  // hopping f^dag_{N,up} f^dag_{N+1,dn} - f^dag_{N,dn} f^dag_{N+1,up}
  for (int i = 0; i < n; ++i)
    for (int j = spsu2_ ? 0 : i + 1; j < n; ++j) {
      if (i == j) continue;
      for (int ch = 0; ch < P_; ++ch) {
        // sum over spin of f^dag_{N,ch,sigma} f_{N+1,ch,sigma}: the site's
        // annihilator is the transpose of its creation operator
        const double v = elem(i, S, S, j, S, S, 0.5, 0.5, &cd_[2 * ch], true, true) +
                         elem(i, S, S, j, S, S, 0.5, -0.5, &cd_[2 * ch + 1], true, true);
        if (fabs(v) > 1e-13) out.push_back({i + 1, j + 1, ch, v, 0});
      }
    }
  if (spsu2_) {
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        if (i == j) continue;
        for (int ch = 0; ch < P_; ++ch) {
          const double v = elem(i, S, S, j, S, S, 0.5, 0.5, &cd_[2 * ch + 1], false, true) -
                           elem(i, S, S, j, S, S, 0.5, -0.5, &cd_[2 * ch], false, true);
          if (fabs(v) > 1e-13) out.push_back({i + 1, j + 1, ch, v, 1});
        }
      }
    // on-site pairing between combinations of one ancestor, in units of
    // 2 delta; the reference writes the pairing of the odd channels with the
    // opposite sign along the chain and its tables with the opposite sign to
    // match (initial.m, bcsgap section).  The element does not depend on the
    // subspace; it is taken at S = 2.
    for (int ch = 0; ch < P_; ++ch)
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
          if (combos_[i].In != combos_[j].In) continue;
          const double v = elem(i, 2.0, 2.0, j, 2.0, 2.0, -1.0, 0.0, &pair_[ch], false, false);
          if (fabs(v) > 1e-13) out.push_back({i + 1, j + 1, ch, (ch % 2 == 0 ? 0.5 : -0.5) * v, 2});
        }
  }
  return off_[ss] = out;
}

const std::vector<RecalcTable>& QSCoupling::recalc_f(const Invar& Ip) {
  auto it = rf_.find(Ip);
  if (it != rf_.end()) return it->second;
  std::vector<RecalcTable> out;
  for (int dss : {1, -1}) {
    const Invar I1{spsu2_ ? 0 : Ip.first + 1, Ip.second + dss};
    if (I1.second < 1) continue;
    for (int ch = 0; ch < P_; ++ch) {
      RecalcTable t{I1, ch, {}};
      for (int i1 = 0; i1 < combs(); ++i1)
        for (int ip = 0; ip < combs(); ++ip) {
          const Invar A = anc(i1, I1);
          if (A != anc(ip, Ip) || A.second < 1) continue;
          const double v = reduced(I1, Ip, 0.5, [&](double q, double S1, double Sp, double M2) {
            return elem(i1, S1, S1, ip, Sp, M2, -1.0, 0.0, &cd_[2 * ch + (q > 0 ? 0 : 1)], false, false);
          });
          if (fabs(v) > 1e-13) t.rows.push_back({i1 + 1, ip + 1, v});
        }
      out.push_back(t);
    }
  }
  return rf_[Ip] = out;
}

std::vector<RecalcRow> QSCoupling::chain_op(const Invar& I1, const Invar& Ip, double rank, bool odd) const {
  std::vector<RecalcRow> rows;
  for (int i1 = 0; i1 < combs(); ++i1)
    for (int ip = 0; ip < combs(); ++ip) {
      if (mult_key(combos_[i1]) != mult_key(combos_[ip])) continue;
      if (anc(i1, I1).second < 1 || anc(ip, Ip).second < 1) continue;
      const double v = reduced(I1, Ip, rank, [&](double q, double S1, double Sp, double M2) {
        return elem(i1, S1, S1, ip, Sp, M2, rank, q, nullptr, false, odd);
      });
      if (fabs(v) > 1e-13) rows.push_back({i1 + 1, ip + 1, v});
    }
  return rows;
}

const std::vector<RecalcTable>& QSCoupling::doublet(const Invar& I1) {
  auto it = dbl_.find(I1);
  if (it != dbl_.end()) return it->second;
  std::vector<RecalcTable> out;
  const int q = spsu2_ ? 0 : I1.first - 1;
  const Invar plus{q, I1.second + 1}, minus{q, I1.second - 1};
  out.push_back({plus, 0, chain_op(I1, plus, 0.5, true)});
  if (I1.second > 1) out.push_back({minus, 0, chain_op(I1, minus, 0.5, true)});
  return dbl_[I1] = out;
}

const std::vector<RecalcTable>& QSCoupling::triplet(const Invar& I1) {
  auto it = trp_.find(I1);
  if (it != trp_.end()) return it->second;
  std::vector<RecalcTable> out;
  const Invar same = I1, plus{I1.first, I1.second + 2}, minus{I1.first, I1.second - 2};
  out.push_back({same, 0, chain_op(I1, same, 1.0, false)});
  out.push_back({plus, 0, chain_op(I1, plus, 1.0, false)});
  if (I1.second > 2) out.push_back({minus, 0, chain_op(I1, minus, 1.0, false)});
  return trp_[I1] = out;
}

}  // namespace nrgb
