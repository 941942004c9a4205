#!/usr/bin/env python3
"""Regenerates the golden fixtures in this directory.

Inputs come from the reference's own dataset generator (datagen/gen_dataset.cpp, compiled from the
reference sources into oracle/_ref/gen_dataset by `make -C oracle ref`); expected counts come from
the generator's known answer k = floor(R * pct / 100) capped at S (datagen/gen_dataset.cpp:119-120,
asserted at :209) and from the reference's own CPU join run_sanity_check (src/sanity_check.cpp,
compiled into oracle/_ref/libref_sanity.so). Payloads are the reference's synthesised values
r_val = row + 1, s_val = row + 100000001 (src/hash_kernel.cu:330-336); the oracle's sorted pair
multiset over them is recorded as a digest.

Run from the repository root: python tests/golden/make_golden.py
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as o  # noqa: E402

CASES = [
    # name, R, S, pct, seed, max_pct
    ("g4k_10pct", 4096, 4096, 10.0, 42, None),
    ("g10k_30k_50pct_skew", 10000, 30000, 50.0, 7, 60.0),
    ("g5k_1k_100pct", 5000, 1000, 100.0, 3, None),
    ("g1_1", 1, 1, 100.0, 1, None),
    ("g20k_0pct", 20000, 20000, 0.0, 5, None),
    ("g32k_64k_25pct", 32768, 65536, 25.0, 11, None),
]


def synth_vals(n, base):
    return (np.arange(n, dtype=np.int64) + base).astype(np.uint32)


def main():
    if not (os.path.exists(o.REF_GEN) and o.ref_available()):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    manifest = []
    with tempfile.TemporaryDirectory() as tmp:
        for name, R, S, pct, seed, mx in CASES:
            cmd = [o.REF_GEN, str(R), str(S), str(pct), tmp, str(seed)]
            if mx is not None:
                cmd += ["--max", str(mx)]
            subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
            tag = f"{pct:.1f}" + (f"_max{mx:.1f}" if mx is not None else "")
            rsrc = os.path.join(tmp, f"gen_R{R}_ans{tag}pct.bin")
            ssrc = os.path.join(tmp, f"gen_S{S}_ans{tag}pct.bin")
            shutil.copy(rsrc, os.path.join(HERE, f"{name}_R.bin"))
            shutil.copy(ssrc, os.path.join(HERE, f"{name}_S.bin"))
            rk = np.fromfile(rsrc, dtype=np.uint32)
            sk = np.fromfile(ssrc, dtype=np.uint32)
            k = min(int(R * pct / 100.0), S)
            ref_count, _ = o.ref_count(rk, sk)
            a, b = o.pairs(rk, synth_vals(R, 1), sk, synth_vals(S, 100000001))
            a, b = o.sort_pairs(a, b)
            manifest.append({"name": name, "R": R, "S": S, "pct": pct, "seed": seed, "max_pct": mx,
                             "k": k, "ref_sanity_count": ref_count, "pairs": int(len(a)),
                             "pairs_digest": f"{o.digest(a, b):016x}",
                             "r_file": f"{name}_R.bin", "s_file": f"{name}_S.bin"})
            print(name, k, ref_count, len(a))
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
