"""Extracts the reference's own OpenCL C kernel text for the CPU build under oracle/_ref/ — TEST
INFRASTRUCTURE ONLY.

The reference keeps its device kernels as C# raw string literals:

* `Kernel` in src/TomoStar.Core/Forward/EikonalOpenCl.cs:387-624 (eik_clear, eik_dirty, eik_seed,
  eik_sweep; FP64 under QV_FP64, else times as float pairs hi + lo),
* `Source` and `PairedSource` in src/TomoStar.Core/Numerics/LsqrOpenCl.cs:41-176 (spmv and the vector
  kernels, FP64 and on float pairs).

This script copies each literal out of the reference tree into oracle/_ref/ (git-ignored; nothing of
it is committed) with the two changes the reference's own host makes or OpenCL C needs on a CPU:

1. `{{TOL}}` becomes the settle tolerance as `TryCreate` writes it
   (`SphericalEikonal.SettleTolerance.ToString("R")` = "1E-07", EikonalOpenCl.cs:93);
2. the OpenCL vector literal `(float2)(a, b)` becomes `make_float2(a, b)`: C++ would read the
   parenthesised pair as a comma expression.

Nothing else is touched; `oracle/ref_shim.h` supplies the OpenCL built-ins and `ref_eik.cpp` /
`ref_lsqr.cpp` drive the kernels in the host's order.

    python oracle/ref_extract.py [--root /root/reference] [--out oracle/_ref]
"""
from __future__ import annotations

import argparse
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_ROOT = os.environ.get("TOMOSTAR_REFERENCE", "/root/reference")

# (C# file under the reference root, literal name, output file)
LITERALS = [
    ("src/TomoStar.Core/Forward/EikonalOpenCl.cs", "Kernel", "eik_kernel.cl"),
    ("src/TomoStar.Core/Numerics/LsqrOpenCl.cs", "Source", "lsqr_fp64.cl"),
    ("src/TomoStar.Core/Numerics/LsqrOpenCl.cs", "PairedSource", "lsqr_paired.cl"),
]

# SphericalEikonal.SettleTolerance (SphericalEikonal.cs:332) = 1e-7, formatted by .NET's "R" format
# (shortest round-trip form with a two-digit exponent).
SETTLE_TOLERANCE_R = "1E-07"


def raw_literal(text: str, name: str) -> str:
    """The content of `const string <name> = \"\"\" ... \"\"\";` with C#'s raw-literal indentation rule
    (the closing delimiter's indentation is removed from every line)."""
    m = re.search(r'const\s+string\s+' + re.escape(name) + r'\s*=\s*"""\n(.*?)\n([ \t]*)""";', text, re.S)
    if not m:
        raise SystemExit(f"literal {name} not found")
    body, indent = m.group(1), m.group(2)
    lines = [ln[len(indent):] if ln.startswith(indent) else ln.lstrip(" \t") for ln in body.split("\n")]
    return "\n".join(lines) + "\n"


def convert(src: str) -> str:
    src = src.replace("{{TOL}}", SETTLE_TOLERANCE_R)
    return re.sub(r"\(float2\)\s*\(", "make_float2(", src)


def extract(root: str, out: str) -> list[str]:
    os.makedirs(out, exist_ok=True)
    written = []
    for rel, name, dst in LITERALS:
        with open(os.path.join(root, rel), encoding="utf-8") as f:
            text = f.read()
        body = convert(raw_literal(text, name))
        path = os.path.join(out, dst)
        with open(path, "w") as f:
            f.write(f"// Extracted by oracle/ref_extract.py from {rel} (literal {name}); not committed.\n")
            f.write(body)
        written.append(path)
    return written


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--root", default=DEFAULT_ROOT)
    ap.add_argument("--out", default=os.path.join(HERE, "_ref"))
    args = ap.parse_args()
    for p in extract(args.root, args.out):
        print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
