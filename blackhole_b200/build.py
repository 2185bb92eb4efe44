"""Build the in-tree CUDA library (sm_100a) and, optionally, the CPU oracle.

    python -m blackhole_b200.build           # library only
    python -m blackhole_b200.build --oracle  # library + oracle (+ oracle/_ref when the reference is present)
"""
from __future__ import annotations

import argparse
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent


def build_library(quiet: bool = False) -> Path:
    subprocess.run(["make", "-C", str(PKG / "csrc")], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    return PKG / "lib" / "libblackhole_b200.so"


def build_oracle(quiet: bool = False, ref_src: Path | None = None) -> None:
    """The CPU oracle; with ref_src (the reference's src/ directory) also the
    libraries compiled from the reference's own sources (oracle/_ref)."""
    cmd = ["make", "-C", str(ROOT / "oracle")]
    if ref_src is not None and (Path(ref_src) / "physics" / "kerr.cpp").exists():
        cmd.append(f"REF_SRC={ref_src}")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--ref-src", type=Path, default=None, help="the reference's src/ directory (for oracle/_ref)")
    ap.add_argument("-q", "--quiet", action="store_true")
    a = ap.parse_args()
    print(build_library(a.quiet))
    if a.oracle:
        build_oracle(a.quiet, a.ref_src)


if __name__ == "__main__":
    main()
