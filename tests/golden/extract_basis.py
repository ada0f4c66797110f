"""Copy the H-Ne blocks of a published basis set (Gaussian-94 .gbs, as the
Lightspeed tree ships them under data/basis/) into lightspeed_b200/data/basis/.

The header (the 'cartesian'/'spherical' line and the comment block with the
references) is kept; element blocks after Ne are dropped. Basis-set data are
published tables (EMSL Basis Set Exchange), not code.

  python tests/golden/extract_basis.py NAME [SOURCE_DIR]
      (SOURCE_DIR default: $REFROOT/data/basis, REFROOT default /root/reference)
"""
import os
import sys

_FIRST_ROW = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne"]


def extract(text):
    lines = text.splitlines()
    out = []
    i = 0
    # header: everything up to the first block separator
    while i < len(lines) and lines[i].strip() != "****":
        out.append(lines[i])
        i += 1
    out.append("****")
    i += 1
    while i < len(lines):
        # a block: element line, shells, then a '****' line
        j = i
        while j < len(lines) and lines[j].strip() != "****":
            j += 1
        block = lines[i:j]
        head = block[0].split() if block else []
        if head and head[0] in _FIRST_ROW:
            out.extend(block)
            out.append("****")
        i = j + 1
    return "\n".join(out) + "\n"


def main():
    name = sys.argv[1]
    src_dir = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.environ.get("REFROOT", "/root/reference"),
                                                                 "data", "basis")
    with open(os.path.join(src_dir, name + ".gbs")) as fh:
        text = fh.read()
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "lightspeed_b200", "data", "basis",
                       name + ".gbs")
    with open(dst, "w") as fh:
        fh.write(extract(text))
    print("wrote", os.path.normpath(dst))


if __name__ == "__main__":
    main()
