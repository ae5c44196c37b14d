"""Golden values of the 'He2S_fci' pair potential (Select_Pot entry of the
reference, V_impur.f90:179-183 and 2962-3008).

Reads the Pg constants of Block Data Inicio_LJ_V_He2s_fci as text from the
reference's V_impur.f90 and evaluates V(x) = sum_{k=1..11} Pg(k) x^-(5+k)
exactly in rational arithmetic (fractions.Fraction of the decimal
constants), rounded once to double, at a set of radii.  The reference sums
in real*16; its result rounded to double agrees with the exact value to
within one double ulp, which is what the oracle test allows.  Run once in a
checkout that has the reference sources; the JSON is committed.

Usage: python make_he2s.py /path/to/reference/V_impur.f90
       (or set HE4_REFERENCE_DIR to the reference checkout)
"""
import json
import os
import re
import sys
from fractions import Fraction


def main():
    if len(sys.argv) > 1:
        src = sys.argv[1]
    elif os.environ.get("HE4_REFERENCE_DIR"):
        src = os.path.join(os.environ["HE4_REFERENCE_DIR"], "V_impur.f90")
    else:
        sys.exit("usage: make_he2s.py <path of the reference's V_impur.f90>")
    txt = open(src, encoding="latin-1").read()
    blk = txt[txt.index("Block Data Inicio_LJ_V_He2s_fci"):]
    body = re.search(r"Data Pg/(.*?)/", blk, re.S).group(1)
    pg = [v.replace("&", "").strip().replace("Q0", "") for v in body.replace("\n", " ").split(",")]
    pg = [v for v in pg if v]
    assert len(pg) == 11
    k0 = int(re.search(r"Data k0/\s*(\d+)", blk).group(1))
    rcut = float(re.search(r"Data rcutoff/\s*([0-9.D+-]+)", blk).group(1).replace("D", "E"))
    fcut = float(re.search(r"Data fcutoff/\s*([0-9.D+-]+)", blk).group(1).replace("D", "E"))
    radii = [3.17502, 3.175021, 3.2, 3.3, 3.5, 3.75, 4.0, 4.5, 5.0, 6.0, 7.5, 10.0, 15.0, 25.0, 60.0, 200.0]
    vals = []
    for x in radii:
        if x <= rcut:
            v = fcut
        else:
            q = Fraction(1) / Fraction(x)
            v = float(sum(Fraction(c) * q ** (k0 + 1 + k) for k, c in enumerate(pg)))
        vals.append(v.hex())
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "he2s_fci.json"), "w") as f:
        json.dump({"source": "V_impur.f90 Block Data Inicio_LJ_V_He2s_fci, V_He2s_fci", "pg": pg, "k0": k0,
                   "rcutoff": rcut, "fcutoff": fcut, "r": radii, "v": vals}, f, indent=1)
    print(f"wrote {len(radii)} values")


if __name__ == "__main__":
    main()
