"""Make the reference's own Python package importable in this container.

TEST INFRASTRUCTURE ONLY (fixture generation and oracle validation). Nothing
on the GPU side imports this module: the reference tree is not present there.

Three shims stand in for what the reference needs and this image lacks
(``array_api_compat`` -> NumPy, an empty ``spglib``, the package metadata
``hafnium/__init__.py:12`` reads), and ``oracle.kernels`` stands in for the
compiled ``hafnium._kernels`` (the Rust crate cannot be built here).
"""

from __future__ import annotations

import os
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent


def default_reference() -> pathlib.Path | None:
    """The reference tree named by HF_REFERENCE_ROOT, or None when it is unset."""
    root = os.environ.get("HF_REFERENCE_ROOT")
    return pathlib.Path(root) if root else None


def install(reference: pathlib.Path | None = None) -> None:
    """Put the shims and the reference tree on ``sys.path`` and register the kernels."""
    reference = reference or default_reference()
    if reference is None:
        raise FileNotFoundError("no reference tree given (pass it, or set HF_REFERENCE_ROOT)")
    reference = pathlib.Path(reference)
    if not reference.exists():
        raise FileNotFoundError(f"reference tree not found at {reference}")
    shims = str(HERE / "shims")
    if shims not in sys.path:
        sys.path.insert(0, shims)
    if str(reference) not in sys.path:
        # last: the reference tree has its own ``tests`` package, which must not
        # shadow this repository's
        sys.path.append(str(reference))
    if str(HERE.parent) not in sys.path:
        sys.path.insert(0, str(HERE.parent))
    from oracle import kernels

    sys.modules.setdefault("hafnium._kernels", kernels)
