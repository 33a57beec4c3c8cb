"""Test infrastructure: convert the reference's LTC table to raw float32.

Reads ``tabM`` from the reference's ``ltc.inc`` (ltc.inc:2-4, 128*128 entries of a
row-major 3x3 matrix, looked up by material.h:464-476) and writes it as
little-endian float32 [128*128*9].  The output lives under oracle/_ref/ with the
other reference build products; tests feed it to the GPU product so that both
sides importance-sample the specular lobe from the same table.
"""
import re
import sys

import numpy as np


def main(src, dst):
    text = open(src).read()
    start = text.index("tabM[size*size]")
    end = text.index("tabMinv[size*size]")
    body = text[start:end]
    vals = np.array(re.findall(r"-?\d+\.\d+(?:e[-+]?\d+)?", body), dtype=np.float32)
    if vals.size != 128 * 128 * 9:
        raise SystemExit(f"unexpected tabM size {vals.size}")
    vals.astype("<f4").tofile(dst)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
