"""Regenerate dg_tables.inc: the numeric tables the nodal-DG operators are built from.

Two tables must be identical to Apollo's for the right-hand side to agree to
round-off: the triangle cubature rules (points and weights, 15 significant
digits, Apollo src/lib/wxcubaturedata2d.h, selected by cubature order 3(N+1) at
src/lib/wxcubature2d.cc:20-28) and the tabulated warp-and-blend nodes with their
face masks (src/lib/wxpnodaldgfunctions.h:112-256).  Both are published numeric
data; this script only re-emits the numbers, parsed to the nearest double, in
this library's own layout.  It reads the Apollo source tree given on the
command line and is run by hand when the tables change; the build uses the
committed dg_tables.inc.

    python apollo_b200/csrc/gen_tables.py $APOLLO_SRC/lib > apollo_b200/csrc/dg_tables.inc
"""
import re
import sys


def parse_number_block(text):
    return [float(tok) for tok in re.findall(r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?", text)]


def cubature_rules(lib):
    src = open(f"{lib}/wxcubaturedata2d.h").read()
    rules = {}
    for m in re.finditer(r"REAL cub2D_(\d+)\[(\d+)\]\s*=\s*\{\s*//[^\n]*\n(.*?)\};", src, re.S):
        order, n = int(m.group(1)), int(m.group(2))
        vals = parse_number_block(m.group(3))
        assert len(vals) == n, (order, n, len(vals))
        rules[order] = vals
    return rules


def node_sets(lib):
    src = open(f"{lib}/wxpnodaldgfunctions.h").read()
    sets = {}
    for m in re.finditer(r"polyms_Ord_(\d+)\(int po.*?\{(.*?)\n\}", src, re.S):
        N = int(m.group(1))
        body = m.group(2)
        r = parse_number_block(re.search(r"p_r\[\d+\]\s*=\s*\{(.*?)\}", body, re.S).group(1))
        s = parse_number_block(re.search(r"p_s\[\d+\]\s*=\s*\{(.*?)\}", body, re.S).group(1))
        fm = [int(v) for v in re.findall(r"\d+", re.search(r"p_Fmask\[\d+\]\s*=\s*\{(.*?)\}", body, re.S).group(1))]
        Np = (N + 1) * (N + 2) // 2
        assert len(r) == Np and len(s) == Np and len(fm) == 3 * (N + 1), N
        sets[N] = (r, s, fm)
    return sets


def emit(rules, sets):
    out = []
    out.append("// Generated by gen_tables.py: numeric tables for the nodal-DG operators.")
    out.append("// Triangle cubature rules (r, s, w) for cubature order 3(N+1), N = 1..8, and the")
    out.append("// warp-and-blend node sets (r, s) with face masks, N = 1..8.  Values are the")
    out.append("// nearest doubles to Apollo's 15-digit tables (wxcubaturedata2d.h,")
    out.append("// wxpnodaldgfunctions.h); they must match those tables for parity.")
    out.append("#pragma once")
    out.append("namespace apollo_tables {")
    for N in range(1, 9):
        order = 3 * (N + 1)
        vals = rules[order]
        out.append(f"static const int kCubNpts_N{N} = {len(vals)//3};")
        out.append(f"static const double kCubRST_N{N}[{len(vals)}] = {{")
        for i in range(0, len(vals), 3):
            out.append("  " + ", ".join(repr(v) for v in vals[i:i+3]) + ",")
        out.append("};")
    for N in range(1, 9):
        r, s, fm = sets[N]
        out.append(f"static const double kNodeR_N{N}[{len(r)}] = {{" + ", ".join(repr(v) for v in r) + "};")
        out.append(f"static const double kNodeS_N{N}[{len(s)}] = {{" + ", ".join(repr(v) for v in s) + "};")
        out.append(f"static const int kFmask_N{N}[{len(fm)}] = {{" + ", ".join(str(v) for v in fm) + "};")
    out.append("static const double* const kCubRST[9] = {nullptr, kCubRST_N1, kCubRST_N2, kCubRST_N3, kCubRST_N4, kCubRST_N5, kCubRST_N6, kCubRST_N7, kCubRST_N8};")
    out.append("static const int kCubNpts[9] = {0, kCubNpts_N1, kCubNpts_N2, kCubNpts_N3, kCubNpts_N4, kCubNpts_N5, kCubNpts_N6, kCubNpts_N7, kCubNpts_N8};")
    out.append("static const double* const kNodeR[9] = {nullptr, kNodeR_N1, kNodeR_N2, kNodeR_N3, kNodeR_N4, kNodeR_N5, kNodeR_N6, kNodeR_N7, kNodeR_N8};")
    out.append("static const double* const kNodeS[9] = {nullptr, kNodeS_N1, kNodeS_N2, kNodeS_N3, kNodeS_N4, kNodeS_N5, kNodeS_N6, kNodeS_N7, kNodeS_N8};")
    out.append("static const int* const kFmask[9] = {nullptr, kFmask_N1, kFmask_N2, kFmask_N3, kFmask_N4, kFmask_N5, kFmask_N6, kFmask_N7, kFmask_N8};")
    out.append("}  // namespace apollo_tables")
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: gen_tables.py <Apollo src/lib directory>   (e.g. $APOLLO_SRC/lib)")
    lib = sys.argv[1]
    sys.stdout.write(emit(cubature_rules(lib), node_sets(lib)))
