"""Builds and runs the oracle-driven encoder (tests/cpp/oracle_encode.cpp): the
library's host plan + packer with the oracle's CPU brick coder. Test infrastructure."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "_build")
EXE = os.path.join(BUILD, "oracle_encode")
SRCS = [
    os.path.join(ROOT, "tests", "cpp", "oracle_encode.cpp"),
    os.path.join(ROOT, "idx2_b200", "csrc", "format.cpp"),
    os.path.join(ROOT, "idx2_b200", "csrc", "packer.cpp"),
    os.path.join(ROOT, "idx2_b200", "csrc", "zstd_frame.cpp"),
    os.path.join(ROOT, "idx2_b200", "csrc", "encoder.cpp"),
    os.path.join(ROOT, "idx2_b200", "csrc", "dpack_plan.cpp"),
]
ORACLE_C = os.path.join(ROOT, "oracle", "idx2_oracle.c")


def build_oracle_encode() -> str:
    deps = SRCS + [ORACLE_C, os.path.join(ROOT, "tests", "cpp", "dpack_emul.h"),
                   os.path.join(ROOT, "idx2_b200", "csrc", "dpack.h")]
    if os.path.exists(EXE) and all(os.path.getmtime(EXE) >= os.path.getmtime(d) for d in deps):
        return EXE
    os.makedirs(BUILD, exist_ok=True)
    obj = os.path.join(BUILD, "idx2_oracle.o")
    subprocess.run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-c", ORACLE_C, "-o", obj],
                   check=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                    "-I" + os.path.join(ROOT, "idx2_b200", "csrc"), "-I" + os.path.join(ROOT, "oracle"),
                    "-I" + os.path.join(ROOT, "tests", "cpp"), "-pthread"]
                   + SRCS + [obj, "-o", EXE, "-ldl", "-lm"], check=True)
    return EXE


def oracle_encode(raw, dims, dtype, levels, tol, out_dir, name="kat", field="f", brick=(32, 32, 32), chunks=None,
                  dpack=False):
    """chunks: (bricks_per_chunk, chunks_per_file, files_per_dir) or None for the defaults;
    dpack: pack with the device packer's host stages and its kernels restated on the host."""
    exe = build_oracle_encode()
    args = [exe, raw, str(dims[0]), str(dims[1]), str(dims[2]), dtype, str(levels), repr(tol),
            out_dir, name, field] + [str(b) for b in brick]
    if chunks:
        args += [str(c) for c in chunks]
    env = dict(os.environ, ORACLE_DPACK="1" if dpack else "0")
    r = subprocess.run(args, capture_output=True, text=True, env=env)
    return r.returncode, r.stderr
