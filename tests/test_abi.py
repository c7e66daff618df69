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


def test_host_helpers_without_device_fail_loudly(cep):
    """run_population and the deck runner go through the device library only:
    without a GPU they raise, they never fall back to the CPU oracle."""
    if cep.device_count() > 0:
        return
    import importlib

    import numpy as np
    import pytest
    with pytest.raises(cep.CepError) as e:
        cep.run_population("cipa2017", np.zeros(2), np.zeros((2, 20)), bcl=2000.0, dt=0.005, n_pace=1, first_pace=0)
    assert e.value.code == cep.ERR_NO_DEVICE
    deck = importlib.import_module("2ddrugsimulation_b200.deck")
    with pytest.raises(cep.CepError) as e:
        deck.run(deck.read_deck("Simulation_Mode = 1\nBasic_Cycle_Length = 400\nBCL_End = 400\n"))
    assert e.value.code == cep.ERR_NO_DEVICE
