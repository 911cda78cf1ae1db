"""The C ABI library builds, loads and exports everything include/ug.h declares."""

import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header: str) -> list[str]:
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^int\s+(ug_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared("ug.h")
    assert "ug_batch_create" in names and "ug_batch_run" in names and len(names) >= 15


def test_library_exports_every_declared_symbol(ug):
    from ugb200 import _lib

    lib = ctypes.CDLL(_lib.LIB_PATH)
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            for name in declared(h):
                assert hasattr(lib, name), f"{name} declared in include/{h} but not exported"
    assert lib.ug_version() >= 1


def test_invalid_configs_fail_loudly(ug):
    """Configuration errors come back as UG_EINVAL with a message, before any device work."""
    import pytest
    from ugb200 import Packer, UgError, Universe

    for bad in (Universe(dim=4), Universe(T=2), Universe(T=16, terms=20),
                Universe(T=16, terms=5),  # the Philox stream is full band only
                Universe(dim=2, cross1d=1), Universe(round_size=100)):
        with pytest.raises(UgError) as e:
            Packer([bad])
        assert e.value.code == 1 and e.value.args[0]


def test_oracle_library_loads(oracle):
    assert oracle.lib() is not None
