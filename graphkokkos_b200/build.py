"""In-tree build of libgk_b200.so (sm_100a) with make + nvcc."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=None, verbose=False):
    jobs = jobs or max(1, min(8, os.cpu_count() or 1))
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"]
    out = subprocess.run(cmd, capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"building libgk_b200.so failed:\n{out.stdout}\n{out.stderr}")
    return os.path.join(HERE, "lib", "libgk_b200.so")


if __name__ == "__main__":
    print(build(verbose=True))
