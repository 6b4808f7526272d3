"""Generate tests/golden/spsu2_tables.json, spsu2_tables_2ch.json and
spsu2_tables_3ch.json (SS up to 12) from the reference's 1-, 2- and
3-channel SPSU2 coefficient tables
(coefnew/spsu2/spsu2-<P>ch-*.dat, included by src/sym-SPSU2.cc:35-58 and
:120-138 and src/nrg-recalc-SPSU2.cc), evaluated numerically for a range of
spin multiplicities.  Run in a container that has
the reference checkout:

    python tests/golden/make_spsu2_tables.py /root/reference

Same evaluation rules as make_qs_tables.py (S(ss) = (ss-1)/2, Power(a,b) =
a^b; rows that are not finite for a given ss are stored as null).  The
anomalous and isospin-x tables have the layout of the off-diagonal one.
"""
import json
import os
import re
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_qs_tables import _eval, _split_args  # noqa: E402

FILES = ["offdiag", "anomalous", "isospinx", "diag", "spinupa", "spindowna", "doubletp", "doubletm",
         "triplets", "tripletp", "tripletm", "singlet", "In2", "QN"]
FILES_2CH = FILES + ["spinupb", "spindownb"]
FILES_3CH = FILES_2CH + ["spinupc", "spindownc"]


def main(refroot, out, channels=1, files=FILES, ss_max=40):
    base = os.path.join(refroot, "coefnew", "spsu2")
    result = {"ss_range": [1, ss_max], "tables": {}}
    for name in files:
        rows = []
        with open(os.path.join(base, "spsu2-%dch-%s.dat" % (channels, name))) as fh:
            for line in fh:
                line = line.strip()
                if not line:
                    continue
                if name in ("In2", "QN"):
                    m = re.match(r"(In|QN)\[(\d+)\] = Invar\((.*)\);", line)
                    rows.append({"i": int(m.group(2)), "qn": [int(x) for x in _split_args(m.group(3))]})
                    continue
                if name in ("offdiag", "anomalous", "isospinx"):
                    args = _split_args(line[line.index("(") + 1:line.rindex(")")])
                    vals = {ss: _eval(args[3], ss=ss) for ss in range(1, ss_max + 1)}
                    rows.append({"i": int(args[0]), "j": int(args[1]), "ch": int(args[2]), "factor": vals})
                    continue
                if name == "diag":
                    args = _split_args(line[line.index("(") + 1:line.rindex(")")])
                    rows.append({"i": int(args[0]), "ch": int(args[1]), "number": float(args[2])})
                    continue
                args = _split_args(line[line.index("{") + 1:line.rindex("}")])
                if name.startswith("spinup") or name.startswith("spindown"):
                    vals = {ss: _eval(args[2], ssp=ss) for ss in range(1, ss_max + 1)}
                    rows.append({"i1": int(args[0]), "ip": int(args[1]), "factor": vals})
                else:
                    vals = {ss: _eval(args[4], ss1=ss) for ss in range(1, ss_max + 1)}
                    rows.append({"i1": int(args[0]), "ip": int(args[1]),
                                 "IN1_at_ss10": list(_eval(args[2], ss1=10)),
                                 "INp_at_ss10": list(_eval(args[3], ss1=10)), "factor": vals})
        result["tables"][name] = rows
    with open(out, "w") as fh:
        json.dump(result, fh, indent=None, sort_keys=True)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    here = os.path.dirname(os.path.abspath(__file__))
    main(ref, os.path.join(here, "spsu2_tables.json"))
    main(ref, os.path.join(here, "spsu2_tables_2ch.json"), channels=2, files=FILES_2CH)
    main(ref, os.path.join(here, "spsu2_tables_3ch.json"), channels=3, files=FILES_3CH, ss_max=12)
