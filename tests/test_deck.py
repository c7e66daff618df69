"""Reference input decks and Hill files (CEPCell_NEO/modules/commons.cpp,
cipa_drug_bench.cpp) read by 2ddrugsimulation_b200.deck, and the runs a
deck selects (GPU)."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

deck = importlib.import_module("2ddrugsimulation_b200.deck")

DECK = """Simulation_Mode = 3
celltype = 1
NUMBER_OF_PACING = 2
Basic_Cycle_Length = 1000
Time_Step = 0.005abc
Write_Step = 1
Stim_Amplitude = 1.5
Concentrations = 1.25,2.5
Drug_Name = ranolazine
Is_Dutta = 1
Is_Print_Graph
Unknown_Key = 7
"""


def test_defaults_match_set_default_values():
    d = deck.read_deck("")
    assert (d.dt, d.dt_write, d.num_pace1, d.bcl_init, d.bcl_decrement, d.bcl_end) == (0.01, 1.0, 3, 1000.0, 50.0,
                                                                                        2000000.0)
    assert (d.stim_amp, d.stim_dur, d.is_print_graph, d.variant, d.drug_name, d.concs) == (1.0, 0.5, 1, "ori",
                                                                                           "bepridil", "0.0")


def test_deck_parsing_rules():
    d = deck.read_deck(DECK)
    assert d.simulation_mode == 3 and d.celltype == 1.0 and d.num_pace1 == 2  # keys are case-insensitive
    assert d.dt == 0.005                      # strtod parses a prefix
    assert d.stim_amp == 1.5 and d.drug_name == "ranolazine" and d.is_dutta == 1
    assert d.concs == "0,1.25,2.5"            # "0," in front
    assert np.array_equal(deck.concentrations(d), [0.0, 1.25, 2.5])
    # a line with the key alone keeps the previous value (sscanf leaves it)
    assert d.is_print_graph == 1
    assert deck.read_deck("Write_Step = 2\nNumber_of_Pacing\n").num_pace1 == 2
    assert deck.strtol("3.7") == 3 and deck.strtod("x") == 0.0 and deck.strtod(" -1e-3z") == -1e-3
    assert np.array_equal(deck.split_values("0,1,"), [0.0, 1.0, 0.0])  # trailing comma adds a 0


def test_deck_from_a_path_and_a_missing_path(tmp_path):
    f = tmp_path / "deck.txt"
    f.write_text(DECK)
    assert deck.read_deck(f) == deck.read_deck(str(f)) == deck.read_deck(DECK)
    with pytest.raises(FileNotFoundError):
        deck.read_deck(str(tmp_path / "missing_deck.txt"))


def test_long_deck_line_is_read_in_fgets_pieces():
    # 99 characters per fgets piece: the value of an over-long line is cut
    d = deck.read_deck("Drug_Name = " + "x" * 120 + "\n")
    assert d.drug_name == "x" * (99 - len("Drug_Name = "))


def test_hill_csv_and_population_order(tmp_path):
    p = tmp_path / "hill.csv"
    p.write_text("IC50_CaL,h_CaL,IC50_K1,h_K1\n1.5,1.0,2.0,0.8\n3.0,1.1\n")
    h = deck.read_hill_csv(p)
    assert np.array_equal(h, [[1.5, 1.0, 2.0, 0.8], [3.0, 1.1, 2.0, 0.8]])  # short row keeps the tail
    d = deck.read_deck("Concentrations = 1,2\n")
    conc, rows = deck.population(d, h)
    assert np.array_equal(conc, [0, 1, 2, 0, 1, 2])
    assert np.array_equal(rows[:3], np.repeat(h[:1], 3, axis=0)) and np.array_equal(rows[3:], np.repeat(h[1:], 3, 0))
    with pytest.raises(ValueError):
        deck.read_hill_csv("header only\n")


def test_unsupported_modes_are_refused(cep):
    with pytest.raises(cep.CepError):
        deck.run(deck.read_deck("Simulation_Mode = 5\n"))
    d = deck.read_deck("Simulation_Mode = 3\nGNa_Scale = 0.5\nGKs_Scale = 2\n")
    assert d.gna_scale == 0.5 and d.gks_scale == 2.0


@pytest.mark.gpu
def test_deck_runs_match_the_direct_calls(cep, gpu):
    hill = np.zeros((2, 14))
    hill[1, 0::2] = [5.0, 20.0, 40.0, 30.0, 10.0, 50.0, 2.0]
    hill[1, 1::2] = 1.0
    d = deck.read_deck(DECK)
    out = deck.run(d, hill, precision="fp64")
    conc, rows = deck.population(d, hill)
    ref = cep.run_population("ord2011", conc, rows, bcl=1000.0, dt=0.005, n_pace=2, first_pace=1, precision="fp64",
                             celltype=1.0, dutta=True, quirks=False, amp_scale=1.5)
    for k in ("apd90", "apd50", "cad90", "qnet", "vm_peak"):
        assert np.array_equal(out[k], ref[k]), k
    assert (out["status"] == cep.INST_DONE).all() and out["apd90"].shape == (6,)
    # Gna_Scale multiplies GNa after initConsts (cipa_drug_bench.cpp:148)
    d2 = deck.read_deck(DECK + "Gna_Scale = 0.5\n")
    out2 = deck.run(d2, hill, precision="fp64")
    ref2 = cep.run_population("ord2011", conc, rows, bcl=1000.0, dt=0.005, n_pace=2, first_pace=1, precision="fp64",
                              celltype=1.0, dutta=True, quirks=False, amp_scale=1.5, scales={"gna": 0.5})
    assert np.array_equal(out2["dvmdt_max"], ref2["dvmdt_max"])
    assert (out2["dvmdt_max"] < out["dvmdt_max"]).all()
    # Simulation_Mode 1: dynamic restitution of the M cell (celltype 0)
    a = deck.read_deck("Simulation_Mode = 1\nBasic_Cycle_Length = 500\nBCL_End = 300\nBCL_Step = 100\n"
                       "Number_of_Pacing = 4\nTime_Step = 0.02\n")
    r = deck.run(a, precision="fp64")
    b = cep.Batch("tt2004", 1, "fp64")
    b.init(mcell=True)
    r2 = b.restitution([500.0, 400.0, 300.0], 4, 0.02)
    for k in r2:
        assert np.array_equal(r[k], r2[k]), k
