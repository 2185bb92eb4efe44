"""Record the byte layout of the reference's BH_LaunchParams.

Compiles a small C program against the reference's own header
(src/cuda/kernel_launch.h, a plain C header) with the host C compiler and
writes sizeof and every field's offset to launch_params_layout.json, the
fixture tests/test_legacy_layout.py checks include/bh_legacy.h against.
Run from the repository root with the reference checkout given as REF:
    REF=<reference checkout> python tests/golden/make_launch_params_layout.py
"""
import json
import os
import re
import subprocess
import sys
import tempfile
from pathlib import Path

if not os.environ.get("REF"):
    sys.exit("set REF to the reference checkout (the directory holding src/cuda/kernel_launch.h)")
REF = Path(os.environ["REF"])
HERE = Path(__file__).resolve().parent


def fields(header: Path) -> list[str]:
    text = header.read_text()
    body = re.search(r"struct BH_LaunchParams\s*\{(.*?)\};", text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        m = re.search(r"(\w+)\s*(\[\s*\d+\s*\])?\s*$", decl.strip())
        if m and decl.strip():
            names.append(m.group(1))
    return names


def layout(include_dir: Path, header: str, names: list[str]) -> dict:
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{header}"', "int main(void) {",
           '  printf("size %zu\\n", sizeof(struct BH_LaunchParams));']
    src += [f'  printf("{n} %zu\\n", offsetof(struct BH_LaunchParams, {n}));' for n in names]
    src += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "layout.c"
        c.write_text("\n".join(src) + "\n")
        exe = Path(d) / "layout"
        subprocess.run(["gcc", "-std=c99", "-I", str(include_dir), str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    vals = dict(line.split() for line in out.splitlines())
    return {"size": int(vals.pop("size")), "offsets": {k: int(v) for k, v in vals.items()}, "fields": names}


def main() -> int:
    header = REF / "src" / "cuda" / "kernel_launch.h"
    names = fields(header)
    lay = layout(header.parent, "kernel_launch.h", names)
    lay["source"] = "src/cuda/kernel_launch.h struct BH_LaunchParams, gcc -std=c99, x86-64"
    (HERE / "launch_params_layout.json").write_text(json.dumps(lay, indent=1) + "\n")
    print(f"{len(names)} fields, sizeof {lay['size']}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
