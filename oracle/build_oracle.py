"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``flowlenia_oracle.c`` into ``oracle/_build/``:
``liboracle_f32.so`` (float arithmetic in the reference's statement order),
``liboracle_f64.so`` (the FP64 twin) and ``liboracle_f64_noskip.so`` (the FP64
twin without the reintegration's |m| < 1e-10 skip, used only to show where the
reference's mass drift comes from).  ``-ffp-contract=off`` keeps gcc from
fusing multiply-adds, matching Rust, which never contracts.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "flowlenia_oracle.c")
OUT = os.path.join(HERE, "_build")
LIBS = {"f32": os.path.join(OUT, "liboracle_f32.so"), "f64": os.path.join(OUT, "liboracle_f64.so"),
        "f64_noskip": os.path.join(OUT, "liboracle_f64_noskip.so")}
DEFINES = {"f32": [], "f64": ["-DORC_F64"], "f64_noskip": ["-DORC_F64", "-DORC_MASS_SKIP=0"]}


def build(force: bool = False) -> dict:
    os.makedirs(OUT, exist_ok=True)
    for tag, path in LIBS.items():
        if not force and os.path.exists(path) and os.path.getmtime(path) >= os.path.getmtime(SRC):
            continue
        cmd = ["gcc", "-O2", "-std=c11", "-D_GNU_SOURCE", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
               "-fPIC", "-shared", "-fvisibility=hidden", SRC, "-o", path, "-lm"]
        cmd[1:1] = DEFINES[tag]
        subprocess.run(cmd, check=True)
    return dict(LIBS)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
