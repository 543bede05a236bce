import os
import subprocess
import sys

from .. import build as _build

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    exe = os.path.join(HERE, "fp64_peak")
    src = os.path.join(HERE, "fp64_peak.cu")
    if not os.path.exists(exe) or os.path.getmtime(exe) < os.path.getmtime(src):
        subprocess.run([_build.nvcc(), *_build.host_compiler(), *_build.ARCH, "-O3", "-o", exe, src], check=True)
    sys.exit(subprocess.run([exe]).returncode)


if __name__ == "__main__":
    main()
