"""Algorithmic operation counts of the device kernels (roofline numerators).

Counts follow the formulas the kernels evaluate (csrc/chem_warp.cuh,
csrc/linalg_warp.cuh, csrc/bdf_warp.cuh), with add/sub/mul/div and a fused
multiply-add counted as 1/1/1/1/2 flops and exp/log/pow counted separately as
one transcendental each.  Per-cell work of one integration is
    nfe*F_rhs + nje*F_jac + nsetups*(F_M + F_lu) + nni*F_solve + nst*F_step
with the counters the integrator itself reports.
"""
from __future__ import annotations

from typing import Dict

from .workloads import mech_info


def op_counts(mech: str) -> Dict[str, float]:
    info = mech_info(mech)
    n = info["nsp"]
    rhs = 0.0
    tr = 0.0
    jac_extra = 0.0
    ent = 0
    for r in info["reactions"]:
        f = 4 + (r["nf"]) + 2                   # ln kf, kf*prod C, q
        t = 0 if r["constk"] else 1
        if r["rev"]:
            f += 6 + 3 + r["np"] + 1            # sum nu g, ln Kc, kr*prod C, Rf-Rr
            t += 1
        if r["type"] >= 1:
            f += 2 * r["tb"]                    # third-body sum
        if r["type"] >= 2:
            f += 8                              # k0, Pr, blend
            t += 1
        if r["type"] == 3:
            f += 20                             # Fcent, A, B, F
            t += 5 + r["T2"]
        rhs += f
        tr += t
        ent += r["nrow"]
        # Jacobian: derivative pieces + scatter of nrow x (nf + np + tb) entries
        jac_extra += 30 + 2 * r["nrow"] * (r["nf"] + r["np"] + r["tb"])
    species = n * 40.0                          # NASA-7 cp, h, g; concentrations; sums
    gather = 2.0 * ent
    final = 8.0 * n
    F_rhs = species + rhs + gather + final
    F_jac = F_rhs + jac_extra + 3 * 2.0 * ent + n * n * 8.0 + n * n * 2.0
    F_M = 2.0 * n * n
    F_lu = 2.0 / 3.0 * n ** 3
    F_solve = 2.0 * n * n
    F_step = 40.0 * n                           # predict/correct/norms/rescale per step
    return {"F_rhs": F_rhs, "T_rhs": tr, "F_jac": F_jac, "T_jac": tr + 3, "F_M": F_M,
            "F_lu": F_lu, "F_solve": F_solve, "F_step": F_step}


def algorithmic_flops(mech: str, totals: Dict[str, float]) -> float:
    """Flops (transcendentals as one op each) of one batch from total counters."""
    c = op_counts(mech)
    return (totals["total_nfe"] * (c["F_rhs"] + c["T_rhs"])
            + totals["total_nje"] * (c["F_jac"] + c["T_jac"])
            + totals["total_nsetups"] * (c["F_M"] + c["F_lu"])
            + totals["total_nni"] * c["F_solve"]
            + totals["total_nst"] * c["F_step"])


def flops_by_pipe(mech: str, totals: Dict[str, float], mixed: bool):
    """(FP64 flops, FP32 flops) of one batch from total counters.  In the mixed
    form the Newton matrix M = I - gamma J, its LU and the triangular solves run
    in FP32; the RHS, the Jacobian's chain rule (accumulated into the FP32
    matrix) and the step logic stay FP64.  In the FP64 form all of it is FP64."""
    c = op_counts(mech)
    f64 = (totals["total_nfe"] * (c["F_rhs"] + c["T_rhs"])
           + totals["total_nje"] * (c["F_jac"] + c["T_jac"])
           + totals["total_nst"] * c["F_step"])
    lin = totals["total_nsetups"] * (c["F_M"] + c["F_lu"]) + totals["total_nni"] * c["F_solve"]
    return (f64, lin) if mixed else (f64 + lin, 0.0)
