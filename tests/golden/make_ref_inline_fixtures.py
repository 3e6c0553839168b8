"""Builds the pin harness of the reference's inline wavenumber code (oracle/ref_pin, which
includes trunk/lib/four/four_inline.h and trunk/lib/scft/scft_inline.h from the reference tree)
and stores its output as tests/golden/ref_inline.json, the fixture that
tests/test_oracle_ref_inline.py compares the oracle's restatement with.  Needs the reference
tree (default /root/reference, or the REF environment variable) and g++; run from anywhere."""

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    ref = os.environ.get("REF", "/root/reference")
    pin = os.path.join(ROOT, "oracle", "ref_pin")
    subprocess.run(["make", "-C", pin, f"REF={ref}"], check=True)
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "pin_inline")], check=True, capture_output=True,
                         text=True).stdout
    doc = json.loads(out)
    with open(os.path.join(HERE, "ref_inline.json"), "w") as fh:
        json.dump(doc, fh, separators=(",", ":"))
    print(f"{len(doc['cases'])} cases written", file=sys.stderr)


if __name__ == "__main__":
    main()
