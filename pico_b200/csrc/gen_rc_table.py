"""Regenerate p2_rc_table.inc: the Poseidon2-16 round-constant table.

The table is the reference's `RC_16_30_U32` (vm/src/primitives/mod.rs:37-218),
30 rows x 16 raw u32 values, shared by KoalaBear and BabyBear (each field
reduces the raw values mod p, `from_wrapped_u32`, mod.rs:221-240).  The values
are data that must be identical for bit-exact hashes, so they are extracted
verbatim rather than re-derived.

Usage: python gen_rc_table.py <path to reference vm/src/primitives/mod.rs>
"""
import re
import sys
from pathlib import Path


def extract(mod_rs: str):
    text = Path(mod_rs).read_text()
    marker = "RC_16_30_U32: [[u32; 16]; 30] = ["
    start = text.index(marker) + len(marker)
    end = text.index("];", start)
    body = text[start:end]
    nums = [int(x) for x in re.findall(r"\b\d+\b", body)]
    if len(nums) != 30 * 16:
        raise SystemExit(f"expected 480 constants, found {len(nums)}")
    return nums


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python gen_rc_table.py <path to the pico source tree's vm/src/primitives/mod.rs>")
    nums = extract(sys.argv[1])
    out = Path(__file__).with_name("p2_rc_table.inc")
    lines = ["/* Poseidon2-16 raw round constants RC_16_30_U32 (30 rounds x 16 lanes),",
             " * extracted by gen_rc_table.py from the reference's",
             " * vm/src/primitives/mod.rs:37-218.  Each field reduces them mod p. */"]
    for r in range(30):
        row = nums[16 * r:16 * (r + 1)]
        lines.append("{" + ", ".join(f"{v}u" for v in row) + "},")
    out.write_text("\n".join(lines) + "\n")
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
