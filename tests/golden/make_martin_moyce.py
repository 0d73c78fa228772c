"""Writes tests/golden/martin_moyce.json from the reference's own dam-break test.

The reference embeds a digitised Martin & Moyce (1952) dam-break front table in its test
`the_dam_break_front_follows_martin_and_moyce` (src/fluid/step.rs:447-460, `MARTIN_MOYCE`: pairs
of dimensionless time and front position).  It is the only reference-held data on the fluid
path.  This script extracts those pairs from the reference's source so the tests can read them
where the reference tree is absent:

    python tests/golden/make_martin_moyce.py [REFERENCE_ROOT]

REFERENCE_ROOT defaults to /root/reference.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def extract(root: str):
    path = os.path.join(root, "src", "fluid", "step.rs")
    text = open(path).read()
    start = text.index("const MARTIN_MOYCE")
    block = text[start:]
    block = block[: block.index("];")]
    line = text[:start].count("\n") + 1
    pairs = [[float(a), float(b)] for a, b in re.findall(r"\(([0-9.]+),\s*([0-9.]+)\)", block)]
    return pairs, line


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    pairs, line = extract(root)
    out = {
        "source": f"src/fluid/step.rs:{line} (MARTIN_MOYCE, the_dam_break_front_follows_martin_and_moyce)",
        "columns": ["time * sqrt(2 g / width)", "front / width"],
        "pairs": pairs,
    }
    with open(os.path.join(HERE, "martin_moyce.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(f"{len(pairs)} pairs from line {line}")


if __name__ == "__main__":
    main()
