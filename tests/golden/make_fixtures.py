"""Regenerates the golden fixtures under tests/golden/ from the reference tree.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_fixtures.py <reference tree>

It copies the reference's own test data for this path, unchanged in content:
  * data/netlib/*.mps  -> tests/golden/netlib/<name>.mps.gz  (gzip of the file bytes)
  * data/netlib/reference.csv -> tests/golden/netlib/reference.csv (HiGHS 1.15.1 status/objective)
and records each file's SHA-256 in tests/golden/netlib/SHA256SUMS so a test can
check that the fixtures are byte-identical to the reference's data.
"""
import gzip
import hashlib
import os
import shutil
import sys


def main(ref: str) -> None:
    src = os.path.join(ref, "data", "netlib")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "netlib")
    os.makedirs(dst, exist_ok=True)
    sums = []
    for name in sorted(os.listdir(src)):
        path = os.path.join(src, name)
        data = open(path, "rb").read()
        sums.append(f"{hashlib.sha256(data).hexdigest()}  {name}")
        if name.endswith(".mps"):
            with gzip.GzipFile(os.path.join(dst, name + ".gz"), "wb", mtime=0) as f:
                f.write(data)
        else:
            shutil.copyfile(path, os.path.join(dst, name))
    with open(os.path.join(dst, "SHA256SUMS"), "w") as f:
        f.write("\n".join(sums) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <path of the reference source tree>")
    main(sys.argv[1])
