"""Write ref_index.json: the line count of every Python file of a
kemi2805/HLLD-AI checkout, so that tests/test_citations.py can check each
``file.py:a-b`` citation in this repository without the reference present.

    python tests/golden/make_ref_index.py /path/to/HLLD-AI
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(root: str) -> None:
    index = {}
    for sub in ("src", "scripts", "tests"):
        base = os.path.join(root, sub)
        for dirpath, _, files in os.walk(base):
            for f in sorted(files):
                if not f.endswith(".py"):
                    continue
                path = os.path.join(dirpath, f)
                with open(path, encoding="utf-8") as fh:
                    n = sum(1 for _ in fh)
                index[os.path.relpath(path, root)] = n
    out = os.path.join(HERE, "ref_index.json")
    with open(out, "w") as fh:
        json.dump(dict(sorted(index.items())), fh, indent=0)
        fh.write("\n")
    print(f"{len(index)} files -> {out}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_ref_index.py REFERENCE_CHECKOUT")
    main(sys.argv[1])
