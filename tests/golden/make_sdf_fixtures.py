"""Copies two of the reference's SDF field files (data/sdf/yplates1/yplates.dat,
16^3 points, plates normal to y; data/sdf/wall1/wall.dat, 32^3 points, the
field of its wall tests) into tests/golden/sdf/.  Run from the repository
root with the reference tree as the argument:

    python tests/golden/make_sdf_fixtures.py /path/to/reference
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    out = os.path.join(HERE, "sdf")
    os.makedirs(out, exist_ok=True)
    shutil.copyfile(os.path.join(ref, "data", "sdf", "yplates1", "yplates.dat"), os.path.join(out, "yplates.dat"))
    shutil.copyfile(os.path.join(ref, "data", "sdf", "wall1", "wall.dat"), os.path.join(out, "wall.dat"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CTC_REFERENCE", "/root/reference"))
