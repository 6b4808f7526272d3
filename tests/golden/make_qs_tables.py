"""Generate tests/golden/qs_tables.json, qs_tables_2ch.json and
qs_tables_3ch.json from the reference's QS coefficient tables
(coefnew/qs/qs-1ch-*.dat, qs-2ch-*.dat, qs-3ch-*.dat),
evaluated numerically for a range of spin multiplicities.  Run in a container that has the reference checkout:

    python tests/golden/make_qs_tables.py /root/reference

The fixture lets the table tests run where the reference is absent.  Each
table row is evaluated exactly as the reference's C++ would (S(ss) = (ss-1)/2,
Power(a,b) = a^b); rows whose value is not finite for a given ss are stored
as null.
"""
import json
import math
import os
import re
import sys

FILES = ["offdiag", "diag", "spinupa", "spindowna", "doubletp", "doubletm",
         "triplets", "tripletp", "tripletm", "In2", "QN"]


def _ns(**kw):
    ns = {"sqrt": lambda x: math.sqrt(x) if x >= 0 else float("nan"),
          "Power": lambda a, b: a ** b,
          "pow": lambda a, b: a ** b,
          "S": lambda ss: (ss - 1) / 2.0,
          "Invar": lambda *a: tuple(a)}
    ns.update(kw)
    return ns


def _eval(expr, **kw):
    expr = expr.replace("2.*", "2.0*")
    try:
        v = eval(expr, {"__builtins__": {}}, _ns(**kw))
    except ZeroDivisionError:
        return None
    if isinstance(v, float) and not math.isfinite(v):
        return None
    return v


def _split_args(s):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


FILES_2CH = ["offdiag", "diag", "spinupa", "spinupb", "spindowna", "spindownb", "doubletp", "doubletm",
             "triplets", "tripletp", "tripletm", "In2", "QN"]
FILES_3CH = ["offdiag", "diag", "spinupa", "spinupb", "spinupc", "spindowna", "spindownb", "spindownc",
             "doubletp", "doubletm", "triplets", "tripletp", "tripletm", "In2", "QN"]


def main(refroot, out, channels=1, files=FILES, indent=1, ss_max=40):
    base = os.path.join(refroot, "coefnew", "qs")
    result = {"ss_range": [1, ss_max], "tables": {}}
    for name in files:
        path = os.path.join(base, "qs-%dch-%s.dat" % (channels, name))
        rows = []
        with open(path) as fh:
            for line in fh:
                line = line.strip()
                if not line:
                    continue
                if name in ("In2", "QN"):
                    m = re.match(r"(In|QN)\[(\d+)\] = Invar\((.*)\);", line)
                    rows.append({"i": int(m.group(2)), "qn": [int(x) for x in _split_args(m.group(3))]})
                    continue
                if name == "offdiag":
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
                    vals = {ss: _eval(args[4], ss1=ss, q1=0) for ss in range(1, ss_max + 1)}
                    in1 = _eval(args[2], ss1=10, q1=0)
                    inp = _eval(args[3], ss1=10, q1=0)
                    rows.append({"i1": int(args[0]), "ip": int(args[1]),
                                 "IN1_at_q0_ss10": list(in1), "INp_at_q0_ss10": list(inp),
                                 "factor": vals})
        result["tables"][name] = rows
    with open(out, "w") as fh:
        json.dump(result, fh, indent=indent, sort_keys=True)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    here = os.path.dirname(os.path.abspath(__file__))
    main(ref, os.path.join(here, "qs_tables.json"))
    main(ref, os.path.join(here, "qs_tables_2ch.json"), channels=2, files=FILES_2CH, indent=None)
    main(ref, os.path.join(here, "qs_tables_3ch.json"), channels=3, files=FILES_3CH, indent=None, ss_max=14)
