"""Build recipe for the CPU restatement oracle (test infrastructure only):
oracle/qcd_oracle.c -> oracle/liboracle.so."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build():
    src = os.path.join(HERE, "qcd_oracle.c")
    if os.path.exists(LIB) and os.path.getmtime(LIB) > os.path.getmtime(src):
        return LIB
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-o", LIB, src, "-lm"],
                   check=True)
    return LIB


if __name__ == "__main__":
    print(build())
