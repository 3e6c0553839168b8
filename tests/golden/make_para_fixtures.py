"""Copies the reference's three example parameter files (trunk/info/new4.21/{fluid3d,mhd3d,RB}/in/
para.d) into tests/golden/para/ as fixtures, so the para.d reader is tested on them where the
reference tree is absent.  Run once where the reference is mounted:

    python tests/golden/make_para_fixtures.py /root/reference
"""

import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    base = os.path.join(ref_root, "trunk", "info", "new4.21")
    out = os.path.join(HERE, "para")
    os.makedirs(out, exist_ok=True)
    for d in ("fluid3d", "mhd3d", "RB"):
        shutil.copyfile(os.path.join(base, d, "in", "para.d"), os.path.join(out, d + ".para.d"))
        print("wrote", os.path.join(out, d + ".para.d"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
