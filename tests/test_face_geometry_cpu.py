"""Leading-face geometry of the sweep kernels, checked on the CPU: the
device header's face words, mask table and closed-form masks against a
brute-force enumeration of the nine face sites (tests/face_check.cpp)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "pscbfm_b200", "csrc")


def test_face_words_and_masks_match_brute_force(tmp_path):
    exe = str(tmp_path / "face_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-D__host__=", "-D__device__=", "-D__forceinline__=inline",
                    "-I", CSRC, os.path.join(HERE, "face_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 mismatches" in r.stdout
