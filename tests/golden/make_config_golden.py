"""Golden roots of the benchmarked configurations, computed once by the CPU oracle.

The GPU tests (tests/test_gpu_configs.py) and bench.py compare the roots the
CUDA path commits to at full size with these values.  Inputs are the
benchmarks' own: matrix i of a workload is the seeded synthetic matrix with
seed 1000 * base_seed + i (SplitMix64 stream, Monty form), generated here by
the oracle's C generator and on the device by pico_b200.fields.random_matrix_torch
-- the same stream.

Configurations (shapes from bench.py's WORKLOADS):
  single-kb-2^16x64  one 2^16 x 64 KoalaBear trace, log_blowup 1
  uneven-kb-2^30     32 KoalaBear traces, heights 2^10..2^22, widths 8..400,
                     ~2^30 trace cells, log_blowup 1, one mixed-height commit
  recursion-bb-48    48 BabyBear traces, heights 2^8..2^20, widths 4..600,
                     log_blowup 2
  fri-kb-2^23        FRI commit phase of the KoalaBear EF4 codeword that is
                     the coset LDE (log_blowup 1, bit-reversed rows) of a
                     2^22 x 4 seeded matrix (seed 4000), one EF4 element per
                     row; challenger-derived betas; final length 2^0 (the
                     reference's rule) and 2^4

The oracle needs ~45 GB of host memory for recursion-bb-48 (inputs and its
blowup-4 LDEs) and takes minutes per configuration on a few cores.

Usage: python tests/golden/make_config_golden.py [name ...]   (default: all)
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402  (workload shapes and seeds)
from oracle import cpu as orc  # noqa: E402
from pico_b200 import fields as F  # noqa: E402

OUT = Path(__file__).resolve().parent / "config_roots.json"
COMMITS = ("single-kb-2^16x64", "uneven-kb-2^30", "recursion-bb-48")
FRI = "fri-kb-2^23"
FRI_BASE = dict(field=0, log_height=22, width=4, seed=4000, log_blowup=1)


def commit_golden(name: str) -> dict:
    wl = bench.WORKLOADS[name]
    f, b, shapes, seed = wl["field"], wl["log_blowup"], wl["shapes"](), wl["seed"]
    seeds = [seed * 1000 + i for i in range(len(shapes))]
    mats = [orc.random_matrix(f, lh, w, s) for (lh, w), s in zip(shapes, seeds)]
    root, _, _ = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b)
    return {"field": F.NAMES[f], "log_blowup": b, "shapes": [list(s) for s in shapes], "seeds": seeds,
            "trace_cells": int(sum(w << lh for lh, w in shapes)), "root": [int(v) for v in root]}


def fri_golden() -> dict:
    fb = FRI_BASE
    f, b = fb["field"], fb["log_blowup"]
    base = orc.random_matrix(f, fb["log_height"], fb["width"], fb["seed"])
    cw = orc.coset_lde(f, base, b, F.lde_shift(f))
    out = dict(fb)
    for name, lf in (("final_1", 0), ("final_16", 4)):
        roots, betas, final, _ = orc.fri_commit_phase(f, cw, b, lf)
        out[name] = {"log_final_len": lf, "roots": roots.tolist(), "betas": betas.tolist(), "final": final.tolist()}
    return out


def main():
    names = sys.argv[1:] or list(COMMITS) + [FRI]
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    data["generator"] = "tests/golden/make_config_golden.py (CPU oracle, oracle/oracle.c)"
    for name in names:
        t = time.time()
        data[name] = fri_golden() if name == FRI else commit_golden(name)
        print(f"{name}: {time.time() - t:.1f} s", flush=True)
        OUT.write_text(json.dumps(data, indent=1) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
