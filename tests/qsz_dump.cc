// Test harness (built by tests/test_qsz_tables.py): prints the QSZ tables of
// the host's plug-in (host/symmetry.h, SymmetryQSZ) as JSON, one object per
// line, for comparison with the reference's tables.
//   qsz_dump <channels>
#include <cstdio>
#include <cstdlib>

#include "../nrgljubljana-old_b200/host/symmetry.h"

using nrgb::Invar;
using nrgb::RecalcTable;

static void tables(const char* kind, const std::vector<RecalcTable>& ts) {
  printf("{\"kind\":\"%s\",\"tables\":[", kind);
  for (size_t t = 0; t < ts.size(); ++t) {
    printf("%s[[%d,%d],%d,[", t ? "," : "", ts[t].Ip.first, ts[t].Ip.second, ts[t].ch);
    for (size_t r = 0; r < ts[t].rows.size(); ++r)
      printf("%s[%d,%d,%.17g]", r ? "," : "", ts[t].rows[r].i1, ts[t].rows[r].ip, ts[t].rows[r].factor);
    printf("]]");
  }
  printf("]}\n");
}

int main(int argc, char** argv) {
  if (argc != 2) return 2;
  nrgb::SymmetryQSZ S(atoi(argv[1]));
  printf("{\"kind\":\"In\",\"rows\":[");
  for (int i = 0; i < S.combs(); ++i) printf("%s[%d,%d,%d]", i ? "," : "", i + 1, S.In()[i].first, S.In()[i].second);
  printf("]}\n{\"kind\":\"QN\",\"rows\":[");
  for (int i = 0; i < S.combs(); ++i) printf("%s[%d,%d,%d]", i ? "," : "", i + 1, S.QN()[i].first, S.QN()[i].second);
  printf("]}\n{\"kind\":\"offdiag\",\"rows\":[");
  const auto o = S.offdiag({0, 0});
  for (size_t k = 0; k < o.size(); ++k) printf("%s[%d,%d,%d,%.17g]", k ? "," : "", o[k].i, o[k].j, o[k].ch, o[k].factor);
  printf("]}\n{\"kind\":\"diag\",\"rows\":[");
  const auto d = S.diag();
  for (size_t k = 0; k < d.size(); ++k) printf("%s[%d,%d,%.17g]", k ? "," : "", d[k].i, d[k].ch, d[k].number);
  printf("]}\n");
  tables("recalc_f", S.recalc_f({0, 0}));
  tables("doublet", S.recalc_doublet({0, 0}));
  return 0;
}
