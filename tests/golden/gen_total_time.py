"""Copy the reference's own step-counter file into tests/golden/total_time.dat.

    python tests/golden/gen_total_time.py REFERENCE_ROOT
    OBL_REFERENCE_ROOT=... python tests/golden/gen_total_time.py

REFERENCE_ROOT is the root of a checkout of the reference (the directory holding SBL/).

The reference ships readin/total_time.dat (written by output_final, 012_io.f90:485-490,
read by read_flow_field, 102_01_ic.f90:697-705): one list-directed integer.  It is the
only restart-format artefact the reference ships, so it pins the total_time reader and
writer byte for byte.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OBL_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: gen_total_time.py REFERENCE_ROOT (or set OBL_REFERENCE_ROOT)")
    src = os.path.join(root, "SBL", "readin", "total_time.dat")
    shutil.copyfile(src, os.path.join(HERE, "total_time.dat"))
    print("copied", src)
