"""The banded nearest-direction search of the directional planner against the full search, on
randomised queries over the whole range of candidate-set sizes (tests/nearest_candidate_check.cpp,
compiled here with the planner's own flags)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "nestedcrossapproximation.jl_b200", "csrc")


def test_banded_search_equals_full_search(tmp_path):
    exe = str(tmp_path / "nearest_candidate_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-mfma", "-pthread",
                    "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                    os.path.join(ROOT, "tests", "nearest_candidate_check.cpp"), os.path.join(CSRC, "host_plan.cpp"),
                    "-o", exe], check=True)
    out = subprocess.run([exe, "300"], check=True, capture_output=True, text=True).stdout
    assert out.split()[-1] == "0", out
