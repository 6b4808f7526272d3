"""Generate tests/golden/qsz_tables.json from the reference's 1-, 2- and
3-channel QSZ coefficient tables (coefnew/qsz/qsz-<P>ch-*.dat, included by
src/sym-QSZ.cc:38-60, :133-160 and src/nrg-recalc-QSZ.cc).  Run in a
container that has the reference checkout:

    python tests/golden/make_qsz_tables.py /root/reference

Every QSZ entry is a number (no spin-dependent expression), so each table is
stored once: In2/QN as the combinations' quantum numbers, offdiag and diag
as rows, the <f^dag> tables (spinup*, spindown*) as (i1, ip, factor) rows
and the doublet tables with their ancestor offsets.
"""
import json
import os
import re
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_qs_tables import _eval, _split_args  # noqa: E402

FILES = {1: ["In2", "QN", "offdiag", "diag", "spinupa", "spindowna", "doubletp", "doubletm"],
         2: ["In2", "QN", "offdiag", "diag", "spinupa", "spinupb", "spindowna", "spindownb", "doubletp", "doubletm"],
         3: ["In2", "QN", "offdiag", "diag", "spinupa", "spinupb", "spinupc", "spindowna", "spindownb",
             "spindownc", "doubletp", "doubletm"]}


def main(refroot, out):
    base = os.path.join(refroot, "coefnew", "qsz")
    result = {}
    for P, files in FILES.items():
        tabs = {}
        for name in files:
            rows = []
            with open(os.path.join(base, "qsz-%dch-%s.dat" % (P, name))) as fh:
                for line in fh:
                    line = line.strip()
                    if not line:
                        continue
                    if name in ("In2", "QN"):
                        m = re.match(r"(In|QN)\[(\d+)\] = Invar\((.*)\);", line)
                        rows.append([int(m.group(2))] + [int(x) for x in _split_args(m.group(3))])
                    elif name == "offdiag":  # OFFDIAG(i, j, ch, factor)
                        a = _split_args(line[line.index("(") + 1:line.rindex(")")])
                        rows.append([int(a[0]), int(a[1]), int(a[2]), float(_eval(a[3]))])
                    elif name == "diag":  # DIAG(i, ch, number)
                        a = _split_args(line[line.index("(") + 1:line.rindex(")")])
                        rows.append([int(a[0]), int(a[1]), float(_eval(a[2]))])
                    else:
                        a = _split_args(line[line.index("{") + 1:line.rindex("}")])
                        if name.startswith("spin"):
                            rows.append([int(a[0]), int(a[1]), float(_eval(a[2]))])
                        else:
                            in1 = _eval(a[2], q1=0, ssz1=0)
                            inp = _eval(a[3], q1=0, ssz1=0)
                            rows.append([int(a[0]), int(a[1]), list(in1), list(inp), float(_eval(a[4], q1=0, ssz1=0))])
            tabs[name] = rows
        result[str(P)] = tabs
    with open(out, "w") as fh:
        json.dump(result, fh, indent=None, sort_keys=True)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    main(ref, os.path.join(os.path.dirname(os.path.abspath(__file__)), "qsz_tables.json"))
