"""Builds libswirlc_b200.so in-tree (swirlc_b200/lib) with nvcc for sm_100a.

  python -m swirlc_b200.build [--clean]
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(clean: bool = False, jobs: int = 0) -> str:
  csrc = os.path.join(HERE, 'csrc')
  jobs = jobs or max(2, os.cpu_count() or 2)
  if clean:
    subprocess.run(['make', '-C', csrc, 'clean'], check=True)
  subprocess.run(['make', '-C', csrc, f'-j{jobs}'], check=True)
  return os.path.join(HERE, 'lib', 'libswirlc_b200.so')


if __name__ == '__main__':
  print(build(clean='--clean' in sys.argv))
