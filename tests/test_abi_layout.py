"""The Python binding's structs against include/pico_gpu.h: a small C program
compiled here with the system C compiler prints sizeof and offsetof for
every field the ctypes classes declare, and both layouts must agree (a
mismatch would pass wrong pointers or sizes through the C ABI silently)."""
import ctypes as C
import json
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

# ctypes class name -> C typedef name
STRUCTS = {
    "Matrix": "pico_matrix",
    "Config": "pico_config",
    "Challenger": "pico_challenger",
    "CommitStats": "pico_commit_stats",
    "OpenBatch": "pico_open_batch",
    "FriParams": "pico_fri_params",
    "OpenStats": "pico_open_stats",
    "TraceRef": "pico_trace_ref",
}


def c_layouts(tmp_path: Path) -> dict:
    from pico_b200 import abi

    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "pico_gpu.h"', "int main(void) {",
             '  printf("{");']
    first = True
    for py, cname in STRUCTS.items():
        cls = getattr(abi, py)
        sep = "" if first else ","
        first = False
        lines.append(f'  printf("{sep}\\"{cname}\\": {{\\"size\\": %zu", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf(", \\"{fname}\\": %zu", offsetof({cname}, {fname}));')
        lines.append('  printf("}");')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    subprocess.run([cc, "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


def test_struct_layouts_match_header(tmp_path):
    from pico_b200 import abi

    want = c_layouts(tmp_path)
    for py, cname in STRUCTS.items():
        cls = getattr(abi, py)
        got = {"size": C.sizeof(cls)}
        for fname, _ in cls._fields_:
            got[fname] = getattr(cls, fname).offset
        assert got == want[cname], (py, got, want[cname])


def header_prototypes() -> dict:
    """name -> number of parameters, from the declarations in the header."""
    import re

    text = (ROOT / "include" / "pico_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(pico_gpu_\w+)\s*\(([^;{]*?)\)\s*;", text):
        args = " ".join(m.group(2).split())
        protos[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return protos


def test_binding_argument_counts_match_header():
    from pico_b200 import abi

    protos = header_prototypes()
    assert len(protos) >= 30
    assert set(protos) == set(abi.SIGNATURES)
    for name, n in protos.items():
        assert len(abi.SIGNATURES[name][1]) == n, (name, n, len(abi.SIGNATURES[name][1]))
