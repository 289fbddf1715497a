"""The range allocator behind the library's reserved device regions
(dcsr_b200/csrc/suballoc.hpp), compiled for the CPU with g++ and run:
fixed best-fit / split / merge / region-boundary cases and seeded random
allocation, free and event-completion sequences (tests/cpp/suballoc_test.cpp
checks overlap, alignment, event references and full merging at the end)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_range_allocator(tmp_path):
    exe = str(tmp_path / "suballoc_test")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "dcsr_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "suballoc_test.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"
