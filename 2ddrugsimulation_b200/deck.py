"""Input decks and Hill files of the reference, and the runs they select.

`read_deck` reads a `key = value` input deck as
CEPCell_NEO/modules/commons.cpp:41-256 does: the defaults of
`set_default_values` (:41-80), lines read in 100-byte `fgets` chunks, each
parsed by `sscanf("%s %*s %s")` (the key, a skipped separator token, the
value; a chunk with fewer tokens keeps the previous value), keys compared
case-insensitively, numbers parsed as `strtod` / `strtol` parse a prefix,
and "Concentrations" stored with "0," in front. `read_hill_csv` reads a
Hill file as cipa_drug_bench.cpp:89-100 does (header skipped, rows split on
commas by get_vector_from_string, commons.cpp:258-270).

`run` maps the deck's Simulation_Mode to this library
(CEPCell_NEO/modules/process_bench.cpp:64-130): 1 dynamic restitution
(apdr_bench, TT2004), 2 and 3 the CiPA drug bench on ORd 2011, 33333 the
same bench on ToR-ORd. Other modes raise CepError(ERR_UNSUPPORTED). The
bench always applies the Dutta scaling (cipa_drug_bench.cpp:145 passes
true whatever the mode) and runs the CEPCell_NEO ORd build, which keeps
the requested celltype and scales the intended conductances; `run`
therefore uses this library's ORd with Dutta on and without the
DrugSimulation build's quirks by default. One difference remains: that
build, like DrugSimulation's, leaves PCap, PCaNa and PCaK unblocked when
the Hill row blocks PCa, while the quirk-free form here blocks them too.
Of the deck's conductance scales, these benches apply only Gna_Scale
(CONSTANTS[GNa] *= gna_scale after initConsts, cipa_drug_bench.cpp:148);
`run` does the same. The other G*_Scale keys are read (the ANM benches of
the ten Tusscher models use them) and, as in the reference's drug benches,
have no effect here; Batch.scale applies any of them to a population.
"""
from __future__ import annotations

import dataclasses
import re
from pathlib import Path

import numpy as np

_FLOAT = re.compile(r"\s*([+-]?(?:\d+\.?\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?|inf(?:inity)?|nan))",
                    re.IGNORECASE)
_INT = re.compile(r"\s*([+-]?\d+)")


def strtod(s: str) -> float:
    """C strtod on a prefix: the longest leading number, 0.0 if there is none."""
    m = _FLOAT.match(s)
    return float(m.group(1)) if m else 0.0


def strtol(s: str) -> int:
    """C strtol(s, NULL, 10) on a prefix, 0 if there is none."""
    m = _INT.match(s)
    return int(m.group(1)) if m else 0


@dataclasses.dataclass
class Deck:
    """param_t fields an input deck sets (CEPCell_NEO/modules/param.hpp), with
    the defaults of set_default_values."""
    celltype: float = 0.0
    variant: str = "ori"
    simulation_mode: int = 0
    t_write_vtk: float = 0.0
    num_pace1: int = 3
    bcl_init: float = 1000.0
    dt: float = 0.01
    dt_write: float = 1.0
    stim_amp: float = 1.0
    stim_dur: float = 0.5
    bcl_decrement: float = 50.0
    bcl_end: float = 2000000.0
    bcl_print_start: float = 0.0
    bcl_print_end: float = 0.0
    scaled_gate: int = 0
    drug_name: str = "bepridil"
    concs: str = "0.0"
    gks_scale: float = 1.0
    gkr_scale: float = 1.0
    gcal_scale: float = 1.0
    gna_scale: float = 1.0
    gk1_scale: float = 1.0
    gbna_scale: float = 1.0
    gbca_scale: float = 1.0
    gto_scale: float = 1.0
    gpca_scale: float = 1.0
    gpk_scale: float = 1.0
    gnal_scale: float = 1.0
    is_print_graph: int = 1
    is_dutta: int = 0
    is_using_output: int = 0
    a1656d_mode: int = 0


# deck key (case-insensitive) -> (field, parser)
_KEYS = {
    "celltype": ("celltype", strtod), "variant": ("variant", str), "simulation_mode": ("simulation_mode", strtol),
    "write_time": ("t_write_vtk", strtod), "number_of_pacing": ("num_pace1", strtol),
    "basic_cycle_length": ("bcl_init", strtod), "time_step": ("dt", strtod), "write_step": ("dt_write", strtod),
    "stim_amplitude": ("stim_amp", strtod), "stim_duration": ("stim_dur", strtod),
    "bcl_step": ("bcl_decrement", strtod), "bcl_end": ("bcl_end", strtod),
    "bcl_print_start": ("bcl_print_start", strtod), "bcl_print_end": ("bcl_print_end", strtod),
    "scaled_gate": ("scaled_gate", strtol), "drug_name": ("drug_name", str),
    "gks_scale": ("gks_scale", strtod), "gkr_scale": ("gkr_scale", strtod), "gcal_scale": ("gcal_scale", strtod),
    "gna_scale": ("gna_scale", strtod), "gk1_scale": ("gk1_scale", strtod), "gbna_scale": ("gbna_scale", strtod),
    "gbca_scale": ("gbca_scale", strtod), "gto_scale": ("gto_scale", strtod), "gpca_scale": ("gpca_scale", strtod),
    "gpk_scale": ("gpk_scale", strtod), "gnal_scale": ("gnal_scale", strtod),
    "is_print_graph": ("is_print_graph", strtol), "is_dutta": ("is_dutta", strtol),
    "is_using_output": ("is_using_output", strtol), "a1656d_type": ("a1656d_mode", strtol),
}


def _text(src) -> str:
    """The text of a deck or Hill file given as a path or as its text. A
    single line without "=" or "," is a path, and a missing file raises (the
    reference stops with "Cannot open file", commons.cpp:110-113)."""
    if isinstance(src, Path):
        return src.read_text()
    s = str(src)
    if s and "\n" not in s and "=" not in s and "," not in s:
        return Path(s).read_text()
    return s


def _fgets_chunks(text: str, size: int):
    """The pieces successive fgets(buf, size, fp) calls return."""
    for line in text.splitlines(keepends=True):
        while len(line) > size - 1:
            yield line[: size - 1]
            line = line[size - 1:]
        if line:
            yield line


def read_deck(src) -> Deck:
    """An input deck (a path or its text) as commons.cpp:115-256 reads it."""
    d = Deck()
    key = value = ""
    for chunk in _fgets_chunks(_text(src), 100):
        toks = chunk.split()
        if not toks:
            continue  # sscanf matches nothing; repeating the previous key changes nothing
        key = toks[0]
        if len(toks) >= 3:
            value = toks[2]
        k = key.lower()
        if k == "concentrations":
            d.concs = "0," + value
        elif k in _KEYS:
            field, parse = _KEYS[k]
            setattr(d, field, parse(value))
    return d


def split_values(s: str) -> np.ndarray:
    """get_vector_from_string (commons.cpp:258-270): comma-separated, strtod
    on each piece (a trailing comma adds a 0)."""
    return np.array([strtod(p) for p in s.split(",")], dtype=np.float64)


def concentrations(d: Deck) -> np.ndarray:
    return split_values(d.concs)


def read_hill_csv(src, max_rows: int = 2000) -> np.ndarray:
    """A Hill file as cipa_drug_bench.cpp:89-100 reads it: the header line
    skipped, every later line (150-byte fgets pieces) one row. The bench
    copies each row into one persistent array (:138), so a row shorter than
    the widest keeps the previous row's trailing values (zeros for the
    first)."""
    lines = list(_fgets_chunks(_text(src), 150))[1:]
    rows = [split_values(ln) for ln in lines]
    if not rows or len(rows) > max_rows:
        raise ValueError(f"Hill file must hold 1..{max_rows} rows (has {len(rows)})")
    width = max(len(r) for r in rows)
    out = np.zeros((len(rows), width))
    prev = np.zeros(width)
    for i, r in enumerate(rows):
        prev = prev.copy()
        prev[: len(r)] = r
        out[i] = prev
    return out


def population(d: Deck, hill: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(conc, hill) per instance in the bench's loop order: every sample with
    every concentration of the deck (cipa_drug_bench.cpp:128-146)."""
    concs = concentrations(d)
    hill = np.atleast_2d(np.asarray(hill, np.float64))
    conc = np.tile(concs, len(hill))
    rows = np.repeat(hill, len(concs), axis=0)
    return conc, rows


def run(d: Deck, hill=None, precision: str = "mixed", states_init=None, quirks: bool = False):
    """Run what the deck selects. Returns the restitution records
    (Simulation_Mode 1) or the population biomarkers with the instances'
    (conc, hill) rows (modes 2, 3, 33333)."""
    import importlib
    cep = importlib.import_module("2ddrugsimulation_b200")
    mode = d.simulation_mode
    if mode == 1:  # apdr_bench: 2004_a (M cell) for celltype 0, 2004_b otherwise (apdr_bench.cpp:77-84)
        bcls = cep.apdr_bcls(d.bcl_init, d.bcl_end, d.bcl_decrement)
        b = cep.Batch("tt2004", 1, precision)
        try:
            b.init(mcell=int(np.floor(d.celltype)) == 0)
            return b.restitution(bcls, d.num_pace1, d.dt)
        finally:
            b.close()
    models = {2: "ord2011", 3: "ord2011", 33333: "tomek2019"}
    if mode not in models:
        raise cep.CepError(cep.ERR_UNSUPPORTED, f"Simulation_Mode {mode} is not supported")
    if hill is None:
        raise ValueError("the drug benches need a Hill file")
    if d.is_using_output and states_init is None:
        raise ValueError("Is_Using_Output needs the initial states (output_orudy.dat)")
    conc, rows = population(d, hill)
    n_pace = d.num_pace1
    # the bench evaluates the last 250 paces, and none below 251 paces
    # (cipa_drug_bench.cpp:296); below that the last pace is evaluated here
    first_pace = n_pace - 250 if n_pace > 250 else n_pace - 1
    out = cep.run_population(models[mode], conc, rows, bcl=d.bcl_init, dt=d.dt, n_pace=n_pace,
                             first_pace=first_pace, precision=precision,
                             celltype=d.celltype, dutta=models[mode] == "ord2011", quirks=quirks,
                             dt_write=d.dt_write, amp_scale=d.stim_amp, states_init=states_init,
                             scales={"gna": d.gna_scale} if d.gna_scale != 1.0 else None)
    out["conc"], out["hill"] = conc, rows
    return out
