"""The coarser levels' bands of an encode whose level 0 runs band by band behind the copy of a
host field (idx2_b200/csrc/band_plan.h, used by encode.cu): each brick of level l + 1 runs after
the band holding the last of its children, every brick exactly once, in brick order within its
band (tests/cpp/band_plan_check.cpp, 400 seeded parent maps)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_follow_bands_properties():
    build = os.path.join(HERE, "_build")
    os.makedirs(build, exist_ok=True)
    exe = os.path.join(build, "band_plan_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "idx2_b200", "csrc"),
                    os.path.join(HERE, "cpp", "band_plan_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok 400"), r.stdout + r.stderr
