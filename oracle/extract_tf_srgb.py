"""Build step of the sRGB probe (test infrastructure): copies the reference's
`class TF_SRGB { ... };` verbatim out of pik/color_management.cc into a
header under oracle/_ref/, so that the probe (oracle/srgb_probe.cc)
compiles the reference's own transfer function. color_management.cc as a
whole needs lcms2, which is absent; the class itself needs only
pik/simd/simd.h and pik/rational_polynomial.h.

    python oracle/extract_tf_srgb.py REF_ROOT OUT_HEADER

The output stays in oracle/_ref/ (git-ignored), like the reference's
compiled objects.
"""

from __future__ import annotations

import os
import sys


def extract(source: str, name: str = "TF_SRGB") -> tuple[str, int, int]:
    """Returns (text, first line, last line) of `class <name> { ... };`."""
    lines = source.split("\n")
    start = next(i for i, l in enumerate(lines)
                 if l.startswith(f"class {name} {{"))
    depth = 0
    for i in range(start, len(lines)):
        depth += lines[i].count("{") - lines[i].count("}")
        if depth == 0 and lines[i].rstrip().endswith("};"):
            return "\n".join(lines[start:i + 1]), start + 1, i + 1
    raise ValueError(f"class {name}: no closing brace")


def main(ref_root: str, out: str) -> None:
    path = os.path.join(ref_root, "pik", "color_management.cc")
    with open(path) as f:
        text, first, last = extract(f.read())
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    with open(out, "w") as f:
        f.write(f"// Extracted from pik/color_management.cc:{first}-{last} "
                f"by oracle/extract_tf_srgb.py.\n")
        f.write(text + "\n")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
