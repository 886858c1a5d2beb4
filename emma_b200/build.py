"""Build libemmahydro.so (sm_100a) and the oracle libraries in-tree with make."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(jobs=8, with_oracle=True):
    subprocess.run(["make", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    if with_oracle:
        subprocess.run(["make", "-j", str(jobs), "-C", os.path.join(ROOT, "oracle")], check=True)
    return os.path.join(HERE, "libemmahydro.so")


if __name__ == "__main__":
    print(build())
