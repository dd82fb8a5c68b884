"""Build the in-tree CUDA library (sm_100a) with the Makefile in csrc/."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=8):
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    return os.path.join(HERE, "lib", "libcoolbubble_b200.so")


if __name__ == "__main__":
    print(build())
