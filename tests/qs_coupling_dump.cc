// Test harness (built by tests/test_qs_coupling_cpp.py): prints the QS
// tables of the host's C++ derivation (host/qs_coupling.cc) as JSON, one
// object per line, for comparison with the oracle's Python derivation.
//   qs_coupling_dump <channels> <largest SS>
#include <cstdio>
#include <cstdlib>

#include "../nrgljubljana-old_b200/host/qs_coupling.h"

using nrgb::Invar;
using nrgb::RecalcTable;

static void rows(const std::vector<RecalcTable>& ts) {
  printf("[");
  for (size_t t = 0; t < ts.size(); ++t) {
    printf("%s[[%d,%d],%d,[", t ? "," : "", ts[t].Ip.first, ts[t].Ip.second, ts[t].ch);
    for (size_t r = 0; r < ts[t].rows.size(); ++r)
      printf("%s[%d,%d,%.17g]", r ? "," : "", ts[t].rows[r].i1, ts[t].rows[r].ip, ts[t].rows[r].factor);
    printf("]]");
  }
  printf("]");
}

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  const int P = atoi(argv[1]), ssmax = atoi(argv[2]);
  nrgb::QSCoupling C(P);
  printf("{\"kind\":\"diag\",\"rows\":[");
  const auto d = C.diag();
  for (size_t k = 0; k < d.size(); ++k) printf("%s[%d,%d,%.17g]", k ? "," : "", d[k].i, d[k].ch, d[k].number);
  printf("]}\n");
  for (int ss = 1; ss <= ssmax; ++ss) {
    printf("{\"kind\":\"offdiag\",\"ss\":%d,\"rows\":[", ss);
    const auto& o = C.offdiag(ss);
    for (size_t k = 0; k < o.size(); ++k)
      printf("%s[%d,%d,%d,%.17g]", k ? "," : "", o[k].i, o[k].j, o[k].ch, o[k].factor);
    printf("]}\n");
  }
  for (int q = -1; q <= 1; ++q)
    for (int ss = 1; ss <= ssmax; ++ss) {
      const Invar I{q, ss};
      printf("{\"kind\":\"recalc_f\",\"I\":[%d,%d],\"tables\":", q, ss);
      rows(C.recalc_f(I));
      printf("}\n{\"kind\":\"doublet\",\"I\":[%d,%d],\"tables\":", q, ss);
      rows(C.doublet(I));
      printf("}\n{\"kind\":\"triplet\",\"I\":[%d,%d],\"tables\":", q, ss);
      rows(C.triplet(I));
      printf("}\n");
    }
  return 0;
}
