"""Regenerates the golden fixtures in this directory.

Run it from the repository root where the reference tree is available:

    python tests/golden/make_fixtures.py [/path/to/reference]

It writes two kinds of files:

* inputs restated here: the clist and bulk test particles of
  src/test/clist/{0,1,2}/main and src/test/bulk/{0,1}/main
  made the way pre/units/gen_random.cpp makes them (drand48 from its
  unseeded glibc state, ``L*(-0.5f + 0.9999f*drand48())`` in double, stored as
  float, printed with ``%f``).  When ``oracle/_ref/gen_random`` (the reference
  generator built from its own sources by oracle/ref.mk) exists, its output
  must be byte-identical;
* the reference's own golden outputs and mesh/particle data, copied verbatim
  (src/test_data/*.txt, src/data/pair/2, src/data/cells/rbc/*.off).
"""
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# src/test/clist/{0,1,2}/main: generator box (X, Y, Z), N; the clist box is 4x6x8
CLIST_CASES = {
    "t0": ((4, 6, 8), 128),
    "t1": ((2, 6, 8), 64),
    "t2": ((20, 6, 8), 64),
}

# src/test/bulk/{0,1}/main: gen_random box and N (the bulk box is the same)
BULK_CASES = {
    "t0": ((4, 4, 4), 64),
    "t1": ((4, 4, 4), 640),
}

COPIES = {
    "clist.ref.clist.t0.txt": "src/test_data/clist.ref.clist.t0.txt",
    "clist.ref.clist.t1.txt": "src/test_data/clist.ref.clist.t1.txt",
    "clist.ref.clist.t2.txt": "src/test_data/clist.ref.clist.t2.txt",
    "rnd.ref.rnd.t0.txt": "src/test_data/rnd.ref.rnd.t0.txt",
    "pair.ref.pair.0.txt": "src/test_data/pair.ref.pair.0.txt",
    "eng.ref.mesh.eng_kantor.txt": "src/test_data/eng.ref.mesh.eng_kantor.txt",
    "ff.ref.bulk.t0.txt": "src/test_data/ff.ref.bulk.t0.txt",
    "ff.ref.bulk.t1.txt": "src/test_data/ff.ref.bulk.t1.txt",
    "rbc.2562.off": "src/data/cells/rbc/sc/2562.off",
    "pair.in.2.txt": "src/data/pair/2",
    "av.ref.rbc.u.area_volume.dev.0.txt": "src/test_data/av.ref.rbc.u.area_volume.dev.0.txt",
    "rbc.1986.off": "src/data/cells/rbc/1986.off",
    "rbc.642.off": "src/data/cells/rbc/642.off",
    # the disabled rbc.u.simple test's output: positions and forces x 0.1
    # (its pipe through uscale 0.1) of two 642-vertex cells
    "forces.ref.rbc.u.simple.txt": "src/test_data/forces.ref.rbc.u.simple.txt",
}


class Drand48:
    """glibc drand48 from its unseeded state: X0 = 0, X' = a X + c mod 2^48."""

    def __init__(self):
        self.x = 0

    def __call__(self):
        self.x = (0x5DEECE66D * self.x + 0xB) & ((1 << 48) - 1)
        return self.x / float(1 << 48)


def gen_random(X, Y, Z, n):
    """pre/units/gen_random.cpp:16-33 (the srand(12345) call does not seed drand48)."""
    d = Drand48()
    c = float(np.float32(0.9999))
    lines = []
    for _ in range(n):
        vals = [np.float32(L * (-0.5 + c * d())) for L in (X, Y, Z, 2, 2, 2)]
        lines.append(" ".join("%f" % float(v) for v in vals))
    return "\n".join(lines) + "\n"


def main(ref):
    cases = [("clist", name, c) for name, c in CLIST_CASES.items()] + \
        [("bulk", name, c) for name, c in BULK_CASES.items()]
    for kind, name, ((X, Y, Z), n) in cases:
        txt = gen_random(X, Y, Z, n)
        path = os.path.join(HERE, "%s.in.%s.txt" % (kind, name))
        with open(path, "w") as f:
            f.write(txt)
        exe = os.path.join(ROOT, "oracle", "_ref", "gen_random")
        if os.path.exists(exe):
            out = subprocess.run([exe, str(X), str(Y), str(Z), str(n)], capture_output=True,
                                 text=True, check=True).stdout
            if out != txt:
                raise SystemExit("gen_random restatement differs from the reference for " + name)
            print("%s %s: identical to the reference generator" % (kind, name))
    for dst, src in COPIES.items():
        shutil.copyfile(os.path.join(ref, src), os.path.join(HERE, dst))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CTC_REFERENCE", "/root/reference"))
