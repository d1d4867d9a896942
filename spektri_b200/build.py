"""The one build entry: libspektri_b200.so (sm_100a kernels + C ABI) and the
drop-in host binary bin/spektri, compiled in place by nvcc through the
Makefile beside this file, and the CPU checker under oracle/ (test
infrastructure, built so the tests and the CPU baseline can run it).
``__graft_entry__.build()`` and ``python -m spektri_b200.build`` call it.
Imports nothing that needs the built library."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(jobs: int = 8, checker: bool = True) -> None:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", HERE], check=True)
    if checker:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


if __name__ == "__main__":
    build()
