"""Write the basis-set files the J/K tests and benchmarks use into
lightspeed_b200/data/basis/, keeping only the first-row elements H-Ne.

The data are the published basis sets (EMSL/Basis Set Exchange, Gaussian-94
format) as distributed with the Lightspeed reference under data/basis/; this
script copies their H-Ne blocks verbatim so the package does not need the
reference tree at run time.

  python lightspeed_b200/data/extract_basis.py /path/to/reference/data/basis
"""
import os
import re
import sys

NAMES = ["sto-3g", "3-21g", "6-31g", "6-31gs", "6-31gss", "cc-pvdz", "cc-pvdz-minao"]
KEEP = {"H", "HE", "LI", "BE", "B", "C", "N", "O", "F", "NE"}


def extract(src, dst):
    with open(src) as fh:
        lines = fh.readlines()
    out = []
    header_done = False
    block = []
    keep = None
    for line in lines:
        if not header_done:
            # the format line, the reference comments and the first separator
            out.append(line)
            if re.match(r"^\s*\*\*\*\*\s*$", line):
                header_done = True
            continue
        if re.match(r"^\s*\*\*\*\*\s*$", line):
            if keep:
                out.extend(block)
                out.append(line)
            block, keep = [], None
            continue
        if keep is None and re.match(r"^\s*([A-Za-z]+)\s+0\s*$", line):
            keep = line.split()[0].upper() in KEEP
        block.append(line)
    if not out[-1].strip().startswith("****"):
        out.append("****\n")
    with open(dst, "w") as fh:
        fh.writelines(out)


def main():
    src_dir = sys.argv[1]
    dst_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis")
    os.makedirs(dst_dir, exist_ok=True)
    for n in NAMES:
        extract(os.path.join(src_dir, n + ".gbs"), os.path.join(dst_dir, n + ".gbs"))
        print("wrote", n)


if __name__ == "__main__":
    main()
