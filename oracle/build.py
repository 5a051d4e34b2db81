"""Build recipe for the oracle's C restatement (test infrastructure)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(force=False):
    src = os.path.join(HERE, "eac_oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    # -ffp-contract=off keeps every float32 product and sum separately rounded,
    # as in the reference's Numba code.
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                           "-o", out, src])
    return out


if __name__ == "__main__":
    print(build(force=True))
