"""In-place build of libspektri_b200.so and bin/spektri (nvcc, sm_100a)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> None:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", HERE], check=True)


if __name__ == "__main__":
    build()
