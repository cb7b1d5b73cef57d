"""Build libastrofd_b200.so in-tree for sm_100a (``python -m astrofd_b200.build``)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose=False):
    cmd = ["make", "-j4", "-C", os.path.join(HERE, "csrc")]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.check_call(cmd)
    return os.path.join(HERE, "libastrofd_b200.so")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
