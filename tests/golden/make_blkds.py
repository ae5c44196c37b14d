"""Extract the centre rows of the reference's Bickley derivative table.

The reference's BLOCK DATA BLKDS (mates.f:172-14043) holds, for every
npd = M in 3..25 (odd) and derivative order K in 1..M-1, the M x M matrix of
npd-point differentiation weights in the packed layout read by NEWDER with
ICON=1 (newder.f:99-125): for K < M-1 only the first (M*M+1)/2 entries are
stored and the rest follow by the symmetry DKF(M*M-J+1) = (-1)^K DKF(J); for
K = M-1 one row of M entries is stored and repeated.  The periodic
derivatives (icon=8) use only the centre row Cdc(K, (M+1)/2, :)
(init_deriv_parallel.f90:72-78, 475-650).

This script parses the DATA statements as text, rebuilds the centre rows for
K = 1, 2 and writes them as exact hex floats to blkds_central.json, and the
whole matrices for M = 3..15, K = 1, 2 to blkds_full.json (the icon=12
boundary uses rows 1..M/2 of them, init_deriv_parallel.f90:429-435).  It is
run once, in a checkout that has the reference sources; the JSON is
committed.

Usage: python make_blkds.py /path/to/reference/mates.f
"""
import json
import os
import re
import sys


def parse_table(path):
    lines = open(path, encoding="latin-1").read().splitlines()
    start = next(i for i, l in enumerate(lines) if "BLOCK DATA BLKDS" in l.upper())
    A = {}
    i = start + 1
    head = re.compile(r"DATA\s*\(A\(I\),I=\s*(\d+),\s*(\d+)\)/")
    while i < len(lines):
        l = lines[i]
        if l.strip().upper() == "END":
            break
        m = head.search(l)
        if m:
            lo, hi = int(m.group(1)), int(m.group(2))
            body = l[m.end():]
            j = i + 1
            while "/" not in body:
                body += lines[j][6:]
                j += 1
            body = body.split("/")[0]
            vals = [v.strip() for v in body.split(",") if v.strip()]
            nums = [float(v.upper().replace("D", "E")) for v in vals]
            if len(nums) != hi - lo + 1:
                raise ValueError(f"block {lo}-{hi}: got {len(nums)} numbers")
            for k, v in enumerate(nums):
                A[lo + k] = v
            i = j
        else:
            i += 1
    return A


def first_index(M, K):
    """JI of NEWDER (newder.f:80-92): first table entry for (M, K)."""
    ji = 1
    for I in range(3, M - 1, 2):
        ji += (I * I + 1) * (I - 2) // 2 + I
    ji += ((M * M + 1) // 2) * (K - 1)
    return ji


def matrix(A, M, K):
    """DKF(1..M*M) as NEWDER returns it for ICON=1."""
    m2 = M * M
    half = (m2 + 1) // 2
    ji = first_index(M, K)
    dkf = [0.0] * (m2 + 1)
    if K < M - 1:
        sig = 1.0 - 2.0 * (K % 2)
        for j in range(1, half):
            dkf[j] = A[ji - 1 + j]
            dkf[m2 - j + 1] = sig * A[ji - 1 + j]
        dkf[half] = A[ji - 1 + half]
    else:
        for r in range(M):
            for c in range(M):
                dkf[1 + r * M + c] = A[ji + c]
    return dkf[1:]


def centre_row(A, M, K):
    d = matrix(A, M, K)
    r = M // 2
    return d[r * M:(r + 1) * M]


def main():
    if len(sys.argv) > 1:
        src = sys.argv[1]
    elif os.environ.get("HE4_REFERENCE_DIR"):
        src = os.path.join(os.environ["HE4_REFERENCE_DIR"], "mates.f")
    else:
        sys.exit("usage: make_blkds.py <path of the reference's mates.f> "
                 "(or set HE4_REFERENCE_DIR to the reference checkout)")
    A = parse_table(src)
    out = {}
    for M in range(3, 26, 2):
        for K in (1, 2):
            if K > M - 1:
                continue
            out[f"{M}_{K}"] = [float(v).hex() for v in centre_row(A, M, K)]
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "blkds_central.json"), "w") as f:
        json.dump({"source": "mates.f BLOCK DATA BLKDS (centre rows, K=1,2)", "rows": out}, f, indent=1)
    full = {}
    for M in range(3, 16, 2):
        for K in (1, 2):
            full[f"{M}_{K}"] = [float(v).hex() for v in matrix(A, M, K)]
    with open(os.path.join(here, "blkds_full.json"), "w") as f:
        json.dump({"source": "mates.f BLOCK DATA BLKDS (whole matrices, row-major, K=1,2)", "matrices": full}, f)
    print(f"wrote {len(out)} rows and {len(full)} matrices")


if __name__ == "__main__":
    main()
