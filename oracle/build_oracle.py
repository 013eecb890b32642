"""Builds the oracle's C restatement (oracle/liboracle.so) and, when the
reference tree is present, the reference's own sources (oracle/_ref/).

TEST INFRASTRUCTURE ONLY: the product never links or loads these libraries.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfastrrt_ref.so")


def build_oracle(force=False):
    src = os.path.join(HERE, "fastrrt_oracle.c")
    hdr = os.path.join(HERE, "fastrrt_oracle.h")
    if not force and os.path.exists(ORACLE_SO) and os.path.getmtime(ORACLE_SO) >= max(
            os.path.getmtime(src), os.path.getmtime(hdr)):
        return ORACLE_SO
    # -ffp-contract=off: every float operation rounded on its own (host mode)
    cmd = ["gcc", "-O2", "-std=c11", "-D_POSIX_C_SOURCE=199309L", "-fPIC", "-shared",
           "-ffp-contract=off", "-fopenmp", src, "-o", ORACLE_SO, "-lm"]
    subprocess.check_call(cmd)
    return ORACLE_SO


# Where the reference source tree is read from: $FASTRRT_REFERENCE, else the
# read-only mount this recipe was written against.
DEFAULT_REFERENCE = "/root/reference"


def reference_root():
    """the reference tree to compile from ($FASTRRT_REFERENCE or the default mount)"""
    return os.environ.get("FASTRRT_REFERENCE") or DEFAULT_REFERENCE


def build_ref(reference=None, jobs=8):
    """Compile the reference's sources in place; skipped when the tree is absent
    (the prebuilt library travels with the repository snapshot)."""
    reference = reference or reference_root()
    if not os.path.isdir(os.path.join(reference, "src", "cuda")):
        return REF_SO if os.path.exists(REF_SO) else None
    subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "ref"), f"-j{jobs}",
                           f"REF={reference}"])
    return REF_SO


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_ref())
