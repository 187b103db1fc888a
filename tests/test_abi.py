"""The C ABI library loads and exports every entry point include/hfjk.h declares (CPU).

No compute call is made here: loading needs only the CUDA runtime library.
"""

from __future__ import annotations

import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared(header: str = "hfjk.h") -> list[str]:
    text = (ROOT / "include" / header).read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(hf\w+)\s*\(", text, flags=re.M)))


def all_declared() -> list[str]:
    return sorted({name for h in (ROOT / "include").glob("*.h") for name in declared(h.name)})


def test_header_declares_the_boundary():
    names = declared()
    for name in ("hf_ctx_create", "hf_shells_upload", "hf_build_fitted_tensor", "hf_coulomb", "hf_exchange",
                 "hf_exchange_factored"):
        assert name in names


def test_library_exports_every_declared_symbol():
    from hafnium_b200 import _lib, build

    if not build.LIBRARY.exists():
        pytest.skip("libhfjk.so is not built (python -m hafnium_b200.build)")
    lib = ctypes.CDLL(str(build.LIBRARY))
    missing = [name for name in all_declared() if not hasattr(lib, name)]
    assert not missing, missing
    assert set(declared("hfjk.h")) == set(_lib.EXPORTS)
    assert set(declared("hfbatch.h")) == set(_lib.BATCH_EXPORTS)
    assert len(declared("hfnn.h")) == 8


def test_context_creation_without_a_device_fails_cleanly():
    import torch

    from hafnium_b200 import _lib
    from hafnium_b200.errors import BackendError

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(BackendError):
        _lib.Context(0)
