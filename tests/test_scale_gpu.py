"""Per-instance conductance scaling (cep_batch_scale) against the oracle.

The reference multiplies a conductance constant after initConsts at its
call sites: CONSTANTS[GNa] *= gna_scale in the drug benches
(CEPCell_NEO/modules/cipa_drug_bench.cpp:148, heart.cpp:222) and ten
scale factors per instance in the ten Tusscher population-of-models sweep
(CEP7Cell/modules/population_tn2006.cpp:72-101). The oracle applies the
same products to its constants (cepo_scale); the FP64 GPU path must then
stay within 1e-6 mV of it.
"""
from __future__ import annotations

import numpy as np
import pytest

VM_TOL_FP64 = 1e-6
TT_TEN = ("gks", "gkr", "gk1", "gna", "gbna", "gcal", "gbca", "gto", "gpca", "gpk")


def _trace_vs_oracle(cep, oracle, model, conc, hill, scales, dt, n_steps, bcl, every):
    n = len(conc)
    b = cep.Batch(model, n, "fp64")
    b.init(conc=conc, hill=hill, quirks=True)
    b.set_pacing(bcl)
    for g, f in scales.items():
        b.scale(g, f)
    b.set_protocol(dt, int(np.ceil(n_steps * dt / bcl)) + 1, -1)
    cells = []
    for k in range(n):
        c = oracle.Cell(model, 0.0, conc[k], hill[k], quirks=True)
        c.set_pacing(bcl)
        for g, f in scales.items():
            c.scale(cep.SCALE[g], float(np.broadcast_to(f, (n,))[k]))
        cells.append(c)
    t = 0.0
    err = 0.0
    for _ in range(n_steps // every):
        b.run(every)
        for c in cells:
            c.run(t, dt, every)
        t += every * dt
        v = b.get_states()[:, 0]
        err = max(err, max(abs(v[k] - cells[k].states[0]) for k in range(n)))
    b.close()
    return err, np.array([c.states[0] for c in cells])


@pytest.mark.gpu
def test_tt2006_population_of_models_ten_scales(cep, gpu, oracle):
    """Eight TT2006 instances with the sweep's ten conductance scales drawn
    from its grid (0.25 .. 1.0 in steps of 0.25; g_Ks and g_Kr at 1 as the
    sweep fixes them), one beat at dt = 0.01 ms."""
    rng = np.random.default_rng(31)
    n = 8
    scales = {g: (np.ones(n) if g in ("gks", "gkr") else rng.choice([0.25, 0.5, 0.75, 1.0], n)) for g in TT_TEN}
    conc = np.zeros(n)
    hill = np.zeros((n, 14))
    err, v_end = _trace_vs_oracle(cep, oracle, "tt2006", conc, hill, scales, 0.01, 100000, 1000.0, 5000)
    assert err <= VM_TOL_FP64, err
    # the scales matter: an unscaled cell ends elsewhere
    c = oracle.Cell("tt2006", 0.0, 0.0, hill[0])
    c.set_pacing(1000.0)
    c.run(0.0, 0.01, 100000)
    assert np.abs(v_end - c.states[0]).max() > 1e-3


@pytest.mark.gpu
def test_ord_family_gna_scale_and_others(cep, gpu, oracle):
    """ORd 2011 and CiPA-ORd with GNa (the decks' Gna_Scale) and four more
    conductances scaled per instance: 200 ms at dt = 0.005 ms."""
    rng = np.random.default_rng(32)
    n = 6
    for model, hw in (("ord2011", 14), ("cipa2017", 20)):
        hill = np.zeros((n, hw))
        conc = np.zeros(n)
        scales = {"gna": rng.uniform(0.3, 1.0, n), "gkr": rng.uniform(0.5, 1.5, n), "gcal": rng.uniform(0.5, 1.5, n),
                  "gncx": rng.uniform(0.5, 1.5, n), "pnak": rng.uniform(0.5, 1.5, n)}
        err, _ = _trace_vs_oracle(cep, oracle, model, conc, hill, scales, 0.005, 40000, 1000.0, 4000)
        assert err <= VM_TOL_FP64, (model, err)


@pytest.mark.gpu
def test_scale_rejects_unknown_and_unsupported(cep, gpu):
    b = cep.Batch("ord2011", 4, "fp64")
    b.init()
    with pytest.raises(cep.CepError) as e:
        b.scale("gbna", 2.0)  # ORd's background sodium permeability is a model constant
    assert e.value.code == cep.ERR_UNSUPPORTED
    with pytest.raises(cep.CepError) as e:
        b.scale("gna", [1.0, 1.0, -1.0, 1.0])
    assert e.value.code == cep.ERR_ARG
    assert cep.lib().cep_batch_scale(b._h, 99, np.ones(4).ctypes.data_as(cep._dp)) == cep.ERR_ARG
    b.close()
