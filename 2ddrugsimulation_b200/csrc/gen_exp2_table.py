"""Writes exp2_table.cuh: 2^(j/64) for j = 0..63 as a pair of doubles
(hi = the value rounded to double, lo = the rounded remainder), computed
with 60-digit decimal arithmetic. Used by the FP64 exponential of
cep_device.cuh (a table-driven method after P. T. P. Tang, "Table-driven
implementation of the exponential function in IEEE floating-point
arithmetic", ACM TOMS 15(2), 1989).

    python gen_exp2_table.py   # rewrites exp2_table.cuh beside this file
"""
from __future__ import annotations

from decimal import Decimal, getcontext
from pathlib import Path

N = 64


def table() -> list[tuple[float, float]]:
    getcontext().prec = 60
    out = []
    for j in range(N):
        v = Decimal(2) ** (Decimal(j) / N)
        hi = float(v)  # Decimal -> float rounds to nearest
        lo = float(v - Decimal(hi))
        out.append((hi, lo))
    return out


def constants() -> dict[str, float]:
    getcontext().prec = 60
    ln2 = Decimal(2).ln()
    step = ln2 / N
    l1 = float(step)
    l2 = float(step - Decimal(l1))
    return {"inv_step": float(N / ln2), "step_hi": l1, "step_lo": l2}


def main() -> None:
    rows = table()
    c = constants()
    lines = [
        "// Generated by gen_exp2_table.py: 2^(j/64) = hi + lo for j = 0..63, and",
        "// the reduction constants 64/ln 2 and ln 2/64 = step_hi + step_lo.",
        "#pragma once",
        "",
        "namespace cep {",
        "namespace exp2tab {",
        f"constexpr double kInvStep = {c['inv_step'].hex()};",
        f"constexpr double kStepHi = {c['step_hi'].hex()};",
        f"constexpr double kStepLo = {c['step_lo'].hex()};",
        "__device__ const double2 kTab[64] = {",
    ]
    for j, (hi, lo) in enumerate(rows):
        lines.append(f"    {{{hi.hex()}, {lo.hex()}}},  // j = {j}")
    lines += ["};", "}  // namespace exp2tab", "}  // namespace cep", ""]
    Path(__file__).with_name("exp2_table.cuh").write_text("\n".join(lines))


if __name__ == "__main__":
    main()
