"""Extract the basis-set data this package ships from the reference's bundle.

The reference bundles Basis Set Exchange JSON files (BSD-3-Clause, MolSSI/EMSL;
hafnium/basis/data/README.md) for H-Ar. This script keeps the elements the
water-cluster workloads and the small test molecules use, verbatim per
element, and writes one JSON file per basis set into hafnium_b200/basis_data/.
Run it once where the reference tree is mounted (the path as the argument, or
in HF_REFERENCE_ROOT):

    python tests/golden/extract_basis.py /path/to/reference
"""

from __future__ import annotations

import json
import pathlib
import sys

BASES = ("sto-3g", "cc-pvdz", "def2-universal-jkfit", "def2-svp")
ELEMENTS = ("1", "2", "6", "7", "8")


def main(reference: str) -> None:
    here = pathlib.Path(__file__).resolve().parent.parent.parent / "hafnium_b200" / "basis_data"
    for name in BASES:
        source = pathlib.Path(reference) / "hafnium" / "basis" / "data" / f"{name}.json"
        data = json.loads(source.read_text(encoding="utf-8"))
        kept = {
            "source": "Basis Set Exchange (https://www.basissetexchange.org), BSD-3-Clause; "
            "cite Pritchard et al., J. Chem. Inf. Model. 59, 4814 (2019)",
            "name": name,
            "version": data.get("version"),
            "elements": {
                z: {"electron_shells": data["elements"][z]["electron_shells"]} for z in ELEMENTS
            },
        }
        (here / f"{name}.json").write_text(json.dumps(kept, indent=0), encoding="utf-8")


if __name__ == "__main__":
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HF_REFERENCE_ROOT")
    if not root:
        raise SystemExit("give the reference tree as the argument or in HF_REFERENCE_ROOT")
    main(root)
