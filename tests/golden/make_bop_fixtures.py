"""Copies the small bop fixtures of the reference's post-processing tests
(post/disp/data, post/punto/data/bop) into tests/golden/bop/: the two
text-format files whole, and of the 60,023-particle float file its header and
the first 64 records of its values (1,536 bytes).  Run from the repository
root with the reference tree as the argument:

    python tests/golden/make_bop_fixtures.py /path/to/reference
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    out = os.path.join(HERE, "bop")
    os.makedirs(out, exist_ok=True)
    for f in ("s-00.bop", "s-00.values", "id-00.bop", "id-00.values"):
        shutil.copyfile(os.path.join(ref, "post", "disp", "data", f), os.path.join(out, f))
    src = os.path.join(ref, "post", "punto", "data", "bop")
    for f in ("solvent-00041.bop", "colors_solvent-00041.bop"):
        shutil.copyfile(os.path.join(src, f), os.path.join(out, f))
    with open(os.path.join(src, "solvent-00041.values"), "rb") as fi:
        head = fi.read(64 * 6 * 4)
    with open(os.path.join(out, "solvent-00041.values.head"), "wb") as fo:
        fo.write(head)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CTC_REFERENCE", "/root/reference"))
