"""Build libemmahydro.so (sm_100a) and the oracle libraries in-tree with make.

The oracle's reference libraries (oracle/_ref) compile the reference's own C
sources where its checkout lies: EMMA_REFERENCE_SRC names its src/ folder; when
unset, the checkout's usual location in the build container is used if present.
Without a checkout only the oracle's restatement is built.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DEFAULT_REFERENCE_SRC = "/root/reference/src"


def reference_src():
    src = os.environ.get("EMMA_REFERENCE_SRC") or DEFAULT_REFERENCE_SRC
    return src if os.path.exists(os.path.join(src, "hydro_utils.c")) else None


def build(jobs=8, with_oracle=True):
    subprocess.run(["make", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    if with_oracle:
        cmd = ["make", "-j", str(jobs), "-C", os.path.join(ROOT, "oracle")]
        src = reference_src()
        if src is not None:
            cmd.append(f"REFSRC={src}")
        subprocess.run(cmd, check=True)
    return os.path.join(HERE, "libemmahydro.so")


if __name__ == "__main__":
    print(build())
