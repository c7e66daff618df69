"""The C-ABI library loads and exports every function include/*.h declares
(no compute calls: this runs on CPU-only hosts)."""
from __future__ import annotations

import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(cep_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(cep):
    lib = cep.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert lib.cep_version().decode().startswith("cep_b200")


def test_python_binding_covers_header(cep):
    assert declared_functions() <= set(cep.declared_symbols()) | {"cep_batch_t"}


def test_no_device_fails_loudly(cep):
    if cep.device_count() > 0:
        return
    import pytest
    with pytest.raises(cep.CepError) as e:
        cep.Batch("ord2011", 4)
    assert e.value.code == cep.ERR_NO_DEVICE


def test_server_without_device_fails_loudly(cep):
    if cep.device_count() > 0:
        return
    import pytest
    with pytest.raises(cep.CepError) as e:
        cep.Server("ord2011")
    assert e.value.code == cep.ERR_NO_DEVICE
