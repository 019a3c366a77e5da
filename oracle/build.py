"""Build recipe for the CPU oracle (test infrastructure only).

``build_oracle()`` compiles oracle/sk_oracle.c, sk_oracle_net.c and sk_oracle_mm.c into oracle/liboracle.so with
-ffp-contract=off.  ``build_ref()`` runs oracle/build_ref.sh, which compiles
the sparkit reference from its own sources into oracle/_ref/libsparkit_ref.so
when those sources are present (skipped otherwise).
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsparkit_ref.so")


def build_oracle(force=False):
    src = [os.path.join(HERE, f) for f in ("sk_oracle.c", "sk_oracle_net.c", "sk_oracle_mm.c", "sk_oracle_impl.h",
                                         "sk_oracle_lanczos.h", "sk_oracle.h")]
    if not force and os.path.exists(ORACLE_SO) and all(
        os.path.getmtime(ORACLE_SO) >= os.path.getmtime(s) for s in src
    ):
        return ORACLE_SO
    subprocess.check_call(
        ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
         os.path.join(HERE, "sk_oracle.c"), os.path.join(HERE, "sk_oracle_net.c"), os.path.join(HERE, "sk_oracle_mm.c"),
         "-o", ORACLE_SO, "-lm"]
    )
    return ORACLE_SO


def build_ref():
    subprocess.check_call(["bash", os.path.join(HERE, "build_ref.sh")])
    return REF_SO if os.path.exists(REF_SO) else None


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_ref())
