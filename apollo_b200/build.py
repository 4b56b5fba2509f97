"""Compile libapollo_dg.so (sm_100a) in-tree with nvcc via csrc/Makefile."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    return os.path.join(HERE, "lib", "libapollo_dg.so")


if __name__ == "__main__":
    print(build())
