"""Extract the far-field (|i| >= 32) asymptotic expansions of the lattice Green's
functions into a coefficient table.

The reference ships these expansions as generated C expressions
(src/lgf_3unb0spe.hpp:5-374, one function per kernel).  The values are
mathematical constants of each stencil's lattice Green's function, so the
table has to hold the same numbers; this script turns every expression into a
flat list of monomial terms

    coef * n1^a * n2^b * n3^c * n^e * pi^p        (and coef * log(n) terms)

which ``farfield.json`` stores and which the CUDA setup kernels and the CPU
oracle evaluate with their own code.  It needs the reference sources and sympy,
so it runs only where the reference tree is present; its output is committed.

Usage:  python flups_b200/kernel/gen_farfield.py /path/to/reference/src/lgf_3unb0spe.hpp
"""
import json
import re
import sys
from pathlib import Path

import sympy as sp


def parse_functions(text):
    """Yield (name, dimension, expression string) for every expansion function."""
    pat = re.compile(r"void\s+(\w+)_expansion\(double\*\s*G,([^)]*)\)\s*\{(.*?)\n\}", re.S)
    for m in pat.finditer(text):
        name, args, body = m.group(1), m.group(2), m.group(3)
        ndim = 3 if "n3" in args else 2
        g = re.search(r"G\[0\]\s*=\s*(.*?);\s*$", body, re.S)
        yield name, ndim, g.group(1)


def to_terms(expr_text):
    n1, n2, n3, n = sp.symbols("n1 n2 n3 n", positive=True)
    s = expr_text
    s = re.sub(r"\b(n[123])_(\d+)\b", r"(\1**\2)", s)
    s = s.replace("M_PI", "pi")
    s = re.sub(r"\bpow\(", "Pow(", s)
    expr = sp.sympify(s, locals={"Pow": sp.Pow, "pi": sp.pi, "log": sp.log,
                                 "n1": n1, "n2": n2, "n3": n3, "n": n})
    expr = sp.expand(expr)
    terms, logs = [], []
    for t in sp.Add.make_args(expr):
        coef, rest = t.as_coeff_Mul()
        powers = rest.as_powers_dict()
        e = {"n1": 0, "n2": 0, "n3": 0, "n": 0, "pi": 0}
        has_log = False
        for base, ex in powers.items():
            if base == sp.pi:
                e["pi"] += int(ex)
            elif base == sp.log(n):
                assert ex == 1
                has_log = True
            elif base in (n1, n2, n3, n):
                e[str(base)] += int(ex)
            elif base == 1:
                continue
            else:
                raise ValueError(f"unexpected factor {base}**{ex} in term {t}")
        row = [float(coef), e["n1"], e["n2"], e["n3"], e["n"], e["pi"]]
        (logs if has_log else terms).append(row)
    return terms, logs


def main():
    src = Path(sys.argv[1]).read_text()
    out = {}
    for name, ndim, text in parse_functions(src):
        terms, logs = to_terms(text)
        out[name] = {"ndim": ndim, "terms": terms, "log_terms": logs}
        print(f"{name}: {len(terms)} terms, {len(logs)} log terms", file=sys.stderr)
    dst = Path(__file__).with_name("farfield.json")
    dst.write_text(json.dumps(out, indent=0))
    print(f"wrote {dst}", file=sys.stderr)


if __name__ == "__main__":
    main()
