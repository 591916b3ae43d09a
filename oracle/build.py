"""Build the C restatements of the oracle (TEST INFRASTRUCTURE ONLY).

    python -m oracle.build

Compiles oracle/overlap_oracle.c with gcc into oracle/liboverlap_oracle.so.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, 'liboverlap_oracle.so')
SRC = os.path.join(HERE, 'overlap_oracle.c')


def build_oracle(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + '.tmp'
    subprocess.run(['gcc', '-O2', '-fPIC', '-shared', '-std=c11', '-o', tmp, SRC, '-lm'], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build_oracle(force=True))
