"""Writes reference_constants.json: the operator tables and default constants as the
reference's own source states them, evaluated with Fortran's literal kinds.

    python tests/golden/make_reference_constants.py REFERENCE_DIR

Reads ModOperator.f90 (SBP_operator, :5-121) and ModuleVariables.f90 from the
reference checkout given as the argument and evaluates every literal as the
compiler does: a literal with a D exponent is double precision, any other real
literal is a default (single-precision) real, a quotient of two single-precision
literals is a single-precision division, and a quotient with a double operand is a
double division. The array constructors' values are stored into the REAL(8) tables;
the mirrored bottom blocks follow the loops of ModOperator.f90 (their sign factor and
index formulas are read from the source and checked). Values are written as hex floats.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = re.compile(r"\s*([+-]?)\s*(\d+\.\d*|\.\d+|\d+)([dDeE][+-]?\d+)?\s*")


def literal(text):
    """(value, kind) of one Fortran literal: kind 'd' (REAL(8)), 's' (default REAL) or 'i'."""
    m = NUM.fullmatch(text)
    if not m:
        raise ValueError("not a literal: %r" % text)
    sign, mant, exp = m.groups()
    if exp is None and "." not in mant:
        return int(sign + mant), "i"
    if exp is not None and exp[0] in "dD":
        return float(sign + mant + "e" + exp[1:]), "d"
    return np.float32(sign + mant + ("e" + exp[1:] if exp else "")), "s"


def quotient(text):
    """(value, kind) of literal ( / literal )*, evaluated left to right."""
    parts = text.split("/")
    val, kind = literal(parts[0])
    for p in parts[1:]:
        v2, k2 = literal(p)
        if kind == "s" and k2 == "s":
            val = np.float32(val) / np.float32(v2)
        elif kind == "i" and k2 == "i":
            raise ValueError("integer division in %r" % text)
        else:
            val, kind = float(val) / float(v2), "d"
    return val, kind


def element(text):
    """An array-constructor element, as stored into a REAL(8) table."""
    return float(quotient(text)[0])


def operator_tables(src):
    text = re.sub(r"&\s*\n\s*", "", src)  # join continuation lines
    text = re.sub(r"!.*", "", text)
    tabs = {"SBP1": np.zeros((9, 6)), "SBP2": np.zeros((9, 6)), "TGFILT": np.zeros((9, 11))}
    assign = re.compile(r"\b(SBP1|SBP2|TGfilt|TGFilt)\((\d+),\s*(\d+)(?::(\d+))?\)\s*=\s*(\(/(.*?)/\)|[^\n]+)")
    for m in assign.finditer(text):
        name, row, c0, c1, rhs, inner = m.groups()
        t = tabs[name.upper()]
        vals = [element(e) for e in inner.split(",")] if inner is not None else [element(rhs.strip())]
        c0 = int(c0)
        c1 = int(c1) if c1 is not None else c0
        if len(vals) != c1 - c0 + 1:
            raise ValueError("%s(%s, %d:%d): %d values" % (name, row, c0, c1, len(vals)))
        t[int(row), c0:c1 + 1] = vals
    # bottom blocks: X(i-1,j-1) = f*X(10-i-1, W+1-j-1) for i = 9..6, j = W..1
    mirror = re.compile(r"\b(SBP1|SBP2|TGfilt)\(i-1,j-1\)\s*=\s*([+-]?\d+\.\d*D0)\*\1\(10-i-1,(\d+)-j-1\)")
    found = {}
    for m in mirror.finditer(text):
        found[m.group(1).upper()] = (float(m.group(2).replace("D", "e")), int(m.group(3)))
    for name, width in (("SBP1", 6), ("SBP2", 6), ("TGFILT", 11)):
        f, w1 = found[name]
        if w1 != width + 1:
            raise ValueError("%s mirror index %d" % (name, w1))
        t = tabs[name]
        for i in range(9, 5, -1):
            for j in range(width, 0, -1):
                t[i - 1, j - 1] = f * t[10 - i - 1, w1 - j - 1]
    return tabs


def scalars(src):
    """Initialised REAL / INTEGER declarations of ModuleVariables.f90 whose value is one
    literal: name -> (value, kind)."""
    out = {}
    for line in src.splitlines():
        line = line.split("!")[0]
        if "::" not in line:
            continue
        decl, rest = line.split("::", 1)
        d = decl.strip().upper()
        if not (d.startswith("REAL") or d.startswith("INTEGER") or d.startswith("DOUBLE PRECISION")):
            continue
        for item in re.split(r",(?![^(]*\))", rest):
            if "=" not in item:
                continue
            name, val = (x.strip() for x in item.split("=", 1))
            try:
                v, k = quotient(val)
            except ValueError:
                continue
            if d.startswith("INTEGER"):
                out[name] = (int(v), "i")
            else:
                out[name] = (float(v), k)
    return out


def main(ref):
    with open(os.path.join(ref, "ModOperator.f90")) as f:
        tabs = operator_tables(f.read())
    with open(os.path.join(ref, "ModuleVariables.f90")) as f:
        sc = scalars(f.read())
    real_names = ["gam", "Re", "Pr", "CFL", "sponge_start_top", "sponge_A_top", "sponge_end_left", "sponge_A_left",
                  "C_mu", "C_beta", "C_kappa", "alpha", "sigma_1", "sigma_2", "one_by_h_11", "one_by_h_44",
                  "fourby3", "oneby3", "twoby3"]
    int_names = ["do_viscous_terms", "ShockCapturing", "ControlForcing", "AXIS", "SAT_FARFIELD",
                 "NSCBC_NONREFLECTING", "SAT_NOSLIP_WALL", "NSCBC_NOSLIP_WALL", "SPONGE", "noutput"]
    out = {
        "source": "ModOperator.f90:5-121 (SBP_operator), ModuleVariables.f90 (initialised declarations); "
                  "written by make_reference_constants.py",
        "tables": {k: [[float(x).hex() for x in row] for row in v] for k, v in tabs.items()},
        "reals": {n: {"value": float(sc[n][0]).hex(), "kind": sc[n][1]} for n in real_names},
        "integers": {n: sc[n][0] for n in int_names},
    }
    with open(os.path.join(HERE, "reference_constants.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_constants.py REFERENCE_DIR (the nataraj2/AxisymmetricJet checkout)")
    main(sys.argv[1])
