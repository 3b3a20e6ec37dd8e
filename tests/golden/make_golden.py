"""Regenerate the golden fixtures in tests/golden/.

1. poseidon2_kat.json -- the reference's own known-answer vectors, read as text
   from gnark/poseidon2/poseidon2_koalabear_test.go:61-80 and
   gnark/poseidon2/poseidon2_babybear_test.go:58-77 (zero input state, 16
   canonical outputs).  These pin the permutation to the reference.
2. two_adic.json -- the derived maximal two-adic generators
   (GENERATOR^((p-1)/2^S)); no reference file pins them.
3. oracle_vectors.json -- small seeded cases computed by the C oracle (after
   it reproduces the KATs): permutations, sponge hashes, coset LDEs, mixed
   height commits and FRI commit phases.  They pin the oracle against
   accidental change; the GPU tests compare against the live oracle too.

Usage: python tests/golden/make_golden.py <root of the pico source tree>
"""
from __future__ import annotations

import hashlib
import json
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import cpu as orc  # noqa: E402
from pico_b200 import fields as F  # noqa: E402

OUT = Path(__file__).resolve().parent


def parse_kat(path: Path, marker: str) -> list[int]:
    text = path.read_text()
    i = text.index(marker)
    body = text[i:text.index("}", i)]
    vals = [int(v) for v in re.findall(r'NewFConst\("(\d+)"\)', body)]
    if len(vals) != 16:
        raise SystemExit(f"{path}: expected 16 outputs, found {len(vals)}")
    return vals


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <root of the pico source tree>")
    ref = Path(sys.argv[1])
    kat = {
        "source": "gnark/poseidon2/poseidon2_koalabear_test.go:61-80, gnark/poseidon2/poseidon2_babybear_test.go:58-77",
        "koalabear": {
            "input": [0] * 16,
            "output": parse_kat(ref / "gnark/poseidon2/poseidon2_koalabear_test.go", "expected_output :="),
        },
        "babybear": {
            "input": [0] * 16,
            "output": parse_kat(ref / "gnark/poseidon2/poseidon2_babybear_test.go", "expected_output :="),
        },
    }
    (OUT / "poseidon2_kat.json").write_text(json.dumps(kat, indent=1) + "\n")

    for name, f in (("koalabear", 0), ("babybear", 1)):
        got = orc.permute_canonical(f, np.zeros(16, dtype=np.uint32)).tolist()
        if got != kat[name]["output"]:
            raise SystemExit(f"oracle does not reproduce the {name} KAT; refusing to write vectors")

    two = {
        "koalabear": {"two_adicity": 24, "generator": 3, "max_root": F.two_adic_generator(0, 24)},
        "babybear": {"two_adicity": 27, "generator": 31, "max_root": F.two_adic_generator(1, 27)},
    }
    (OUT / "two_adic.json").write_text(json.dumps(two, indent=1) + "\n")

    vec = {}
    for name, f in (("koalabear", 0), ("babybear", 1)):
        v = {}
        states = F.to_monty(f, F.uniform(f, 4 * 16, 11)).reshape(4, 16)
        v["permute"] = {"seed": 11, "in": states.tolist(), "out": orc.permute(f, states).tolist()}
        hashes = []
        for L in (0, 1, 7, 8, 9, 16, 23):
            x = F.to_monty(f, F.uniform(f, L, 100 + L)) if L else np.zeros(0, dtype=np.uint32)
            hashes.append({"len": L, "seed": 100 + L, "digest": orc.hash_elems(f, x).tolist()})
        v["hash"] = hashes
        ldes = []
        for (logn, w, b, seed) in ((0, 3, 1, 5), (4, 3, 1, 6), (5, 2, 2, 7), (7, 9, 1, 8)):
            m = F.random_matrix(f, logn, w, seed)
            out = orc.coset_lde(f, m, b, F.lde_shift(f))
            ldes.append({"log_n": logn, "width": w, "log_blowup": b, "seed": seed, "sha256": digest(out),
                         "row0": out[0].tolist()})
        v["coset_lde"] = ldes
        shapes = [(5, 3, 21), (5, 5, 22), (3, 2, 23), (1, 7, 24), (5, 0, 25), (0, 4, 26)]
        mats = [F.random_matrix(f, lh, w, s) for lh, w, s in shapes]
        root, _, layers = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), 1, want_layers=True)
        v["pcs_commit"] = {"shapes": shapes, "log_blowup": 1, "root": root.tolist(), "layers_sha256": digest(layers)}
        base = F.random_matrix(f, 5, 4, 31)
        cw = orc.coset_lde(f, base, 1, F.lde_shift(f))
        roots, betas, final, _ = orc.fri_commit_phase(f, cw, 1)
        v["fri"] = {"seed": 31, "log_trace": 5, "log_blowup": 1, "roots": roots.tolist(), "betas": betas.tolist(),
                    "final": final.tolist()}
        vec[name] = v
    (OUT / "oracle_vectors.json").write_text(json.dumps(vec) + "\n")
    print("wrote", [p.name for p in OUT.glob("*.json")])


if __name__ == "__main__":
    main()
