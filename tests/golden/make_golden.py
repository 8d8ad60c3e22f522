"""Regenerates the golden fixtures in this folder.

* murmur3_kat.json — MurmurHash3 known answers computed by the reference's own
  kernels/MurmurHash.cuh, compiled on the host into oracle/_ref/murmur_kat by
  `make -C oracle ref` (needs the reference source tree; REF=<path>).
* tiny_cases.json is hand-written (products worked out by hand) and is not
  regenerated here.

Run: python tests/golden/make_golden.py [REF_PATH]
"""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref", f"REF={ref}"], check=True)
    rng = np.random.default_rng(1234)
    keys = list(range(0, 256)) + [2**k for k in range(8, 32)] + [2**k - 1 for k in range(8, 33)]
    keys += [int(x) for x in rng.integers(0, 2**32, 200, dtype=np.uint64)]
    proc = subprocess.run([str(ROOT / "oracle" / "_ref" / "murmur_kat")], input="\n".join(map(str, keys)) + "\n",
                          capture_output=True, text=True, check=True)
    pairs = [tuple(int(t) for t in line.split()) for line in proc.stdout.strip().splitlines()]
    out = {"source": "reference kernels/MurmurHash.cuh murmurHash3_32, seed MURMUR3_SEED=1234 "
                     "(include/Common.h:73), compiled on the host by oracle/Makefile target 'ref'",
           "seed": 1234, "keys": [k for k, _ in pairs], "hashes": [h for _, h in pairs]}
    (HERE / "murmur3_kat.json").write_text(json.dumps(out) + "\n")
    print(f"wrote {len(pairs)} known answers")


if __name__ == "__main__":
    main()
