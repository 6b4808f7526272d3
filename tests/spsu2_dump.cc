// Test harness (built by tests/test_spsu2_tables.py): prints the SPSU2
// tables of the host's plug-in (host/symmetry.h) as JSON, one object per
// line, for comparison with the oracle's derivation and the reference's
// tables.
//   spsu2_dump <channels> <largest SS>
#include <cstdio>
#include <cstdlib>

#include "../nrgljubljana-old_b200/host/symmetry.h"

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
  nrgb::SymmetrySPSU2 S(P);
  printf("{\"kind\":\"diag\",\"rows\":[");
  const auto d = S.diag();
  for (size_t k = 0; k < d.size(); ++k) printf("%s[%d,%d,%.17g]", k ? "," : "", d[k].i, d[k].ch, d[k].number);
  printf("]}\n");
  for (int ss = 1; ss <= ssmax; ++ss) {
    printf("{\"kind\":\"offdiag\",\"ss\":%d,\"rows\":[", ss);
    const auto o = S.offdiag({0, ss});
    for (size_t k = 0; k < o.size(); ++k)
      printf("%s[%d,%d,%d,%.17g,%d]", k ? "," : "", o[k].i, o[k].j, o[k].ch, o[k].factor, o[k].kind);
    printf("]}\n");
    const Invar I{0, ss};
    printf("{\"kind\":\"recalc_f\",\"I\":[0,%d],\"tables\":", ss);
    rows(S.recalc_f(I));
    printf("}\n{\"kind\":\"doublet\",\"I\":[0,%d],\"tables\":", ss);
    rows(S.recalc_doublet(I));
    printf("}\n{\"kind\":\"triplet\",\"I\":[0,%d],\"tables\":", ss);
    rows(S.recalc_triplet(I));
    printf("}\n");
  }
  return 0;
}
