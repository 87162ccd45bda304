"""PINY's RESPA split of the force path (host side).

PINY integrates with nested RESPA loops (int_NVT_pimd.c:142-223): inter
(``respa_steps_lrf``), torsion, intra and bead levels.  At each inner step it
asks the force routines for one level through the energy_ctrl flags
(int_NVT_pimd.c:175-189) and the routines weight each term by how many inner
steps its impulse spans (energy_control_initial.c:211-243).  The device entry
point ``pinyb200_respa_force_device`` (``DeviceBox.respa_force_device``) takes
the level as a bit set and the split's set-up from ``pinyb200_set_respa``;
this module forms both the way PINY does.
"""
from __future__ import annotations

import numpy as np

FULL_INTER = 1  # energy_ctrl.iget_full_inter
RES_INTER = 2  # energy_ctrl.iget_res_inter
FULL_INTRA = 4  # energy_ctrl.iget_full_intra
RES_INTRA = 8  # energy_ctrl.iget_res_intra


def respa_weights(nres_ter: int, nres_tor: int, nres_tra: int, nres_pimd: int, pimd_on: bool):
    """wght_ter, wght_ter_res, wght_tra_res as energy_control_initial sets
    them (energy_control_initial.c:219-235): integer products of the step
    counts of the levels inside each term's own."""
    if pimd_on:
        return (float(nres_pimd * nres_tra * nres_tor * nres_ter), float(nres_pimd * nres_tra * nres_tor),
                float(nres_pimd))
    return float(nres_tra * nres_tor * nres_ter), float(nres_tra * nres_tor), 1.0


def respa_setup(nres_ter: int, nres_tor: int, nres_tra: int, nres_pimd: int, pimd_on: bool, int_res_ter: bool,
                cutoff_res, rheal_res: float, bond_eq_res, nktot_res: int = 0, ecor_cdv0_res=None, mesh_res=None):
    """Everything pinyb200_set_respa takes: the weights, PINY's switches
    int_res_ter (``respa_steps_lrf`` given), int_res_inter (nres_ter > 1,
    energy_control_initial.c:223-229) and the bond RESPA flag of
    energy_control_intra.c:116-119 (nres_tra*nres_tor > 1), the inner
    cutoffs per pair type (Bohr), the switch width (Bohr), the bonds' RESPA
    equilibrium lengths per bond type (Bohr) and, for the reciprocal-space
    RESPA set on the one PME grid (``ewald_respa_kmax`` = ``ewald_kmax``),
    its k-vector count and the exclusion correction's RESPA force table
    (``system.ecor_res_table``).  ``mesh_res`` -- PINY's separate RESPA PME
    mesh (``ewald_respa_pme_opt on``) as ``system.pme_res_mesh`` returns it:
    ngrid_res, n_interp_res, kastr_res/kbstr_res/kcstr_res, bweight_res."""
    w_ter, w_ter_res, w_tra_res = respa_weights(nres_ter, nres_tor, nres_tra, nres_pimd, pimd_on)
    out = {"wght_ter": w_ter, "wght_ter_res": w_ter_res, "wght_tra_res": w_tra_res,
           "int_res_ter": int(bool(int_res_ter)), "int_res_inter": int(nres_ter > 1),
           "ires_bond": int(nres_tra * nres_tor > 1),
           "cutoff_res": np.ascontiguousarray(cutoff_res, np.float64), "rheal_res": float(rheal_res),
           "bond_eq_res": np.ascontiguousarray(bond_eq_res, np.float64), "nktot_res": int(nktot_res),
           "pme_res_on": 0}
    if ecor_cdv0_res is not None:
        out["ecor_cdv0_res"] = np.ascontiguousarray(ecor_cdv0_res, np.float64)
    if mesh_res is not None:
        out["pme_res_on"] = 1
        out.update(mesh_res)
    return out


def level_bits(iget_full_inter: int, iget_res_inter: int, iget_full_intra: int, iget_res_intra: int) -> int:
    """The level bit set from PINY's four energy_ctrl flags."""
    return ((FULL_INTER if iget_full_inter else 0) | (RES_INTER if iget_res_inter else 0) |
            (FULL_INTRA if iget_full_intra else 0) | (RES_INTRA if iget_res_intra else 0))


def loop_levels(nres_ter: int, nres_tor: int, nres_tra: int, nres_pimd: int, int_res_ter: bool):
    """The level of every force call of one PINY step, in order: int_NVT_pimd's
    four nested loops (int_NVT_pimd.c:142-223) call the force routines when
    ir_pimd == nres_pimd and set the flags as :175-189 does."""
    out = []
    for ir_ter in range(1, nres_ter + 1):
        for ir_tor in range(1, nres_tor + 1):
            for ir_tra in range(1, nres_tra + 1):
                for ir_pimd in range(1, nres_pimd + 1):
                    if ir_pimd != nres_pimd:
                        out.append(0)
                        continue
                    last_tra = ir_tra == nres_tra
                    full_inter = ir_ter == nres_ter and ir_tor == nres_tor and last_tra
                    res_inter = bool(int_res_ter) and ir_tor == nres_tor and last_tra
                    out.append(level_bits(full_inter, res_inter, last_tra, True))
    return out
