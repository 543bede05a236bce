"""Writes tests/golden/formats_ref.txt: the output of tests/cpp/formats.cpp compiled against the
reference's own headers and sources (the compiled reference in oracle/_ref, built by
oracle/Makefile). Run where the reference source tree is present:
    PFSOFT_REFERENCE=<reference source tree> python tests/golden/make_formats.py
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("PFSOFT_REFERENCE", "")


def main() -> int:
    if not REF:
        sys.exit("set PFSOFT_REFERENCE to the reference project's source tree")
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), f"REF={REF}", "ref"], check=True, capture_output=True)
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "formats_ref")
        subprocess.run(["/usr/bin/g++", "-std=c++11", "-O1", "-w", "-fopenmp", "-DUSE_REFERENCE",
                        "-I", os.path.join(ROOT, "oracle", "_ref", "include"), "-I", os.path.join(REF, "include"),
                        os.path.join(ROOT, "tests", "cpp", "formats.cpp"), "-o", exe,
                        "-L", os.path.join(ROOT, "oracle", "_ref"), "-lpfsoft_ref",
                        "-Wl,-rpath," + os.path.join(ROOT, "oracle", "_ref")], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    with open(os.path.join(HERE, "formats_ref.txt"), "w") as f:
        f.write(out)
    print(f"wrote {len(out)} characters")
    return 0


if __name__ == "__main__":
    sys.exit(main())
