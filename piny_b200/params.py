"""Model parameters of q-TIP4P/F as a vector, their tangents, and the
differentiable force call.

theta = (qH [e], gamma [1], sigma [A], epsilon [kcal/mol], D [kcal/mol],
a [1/A], r0 [A], k_bend [kcal/mol/rad^2], theta0 [deg]); the M-site charge is
-2 qH (neutral molecule) and the M site is gamma r_O + (1 - gamma)/2 (r_H1 +
r_H2).  ``tangents`` gives, for every parameter, the exact derivative of the
set-up data `piny_b200.system.build_system` produces (charges, vdW spline
tables, ghost coefficients, bond and bend series, LJ tail), which the
device adjoint (pinyb200_grad) contracts with the force path.

`PinyForceField` evaluates energy and forces of one box for a parameter
vector held in a torch tensor; `EnergyForces` is the torch.autograd.Function
whose backward calls the adjoint, so that dE/dtheta and the gradient of any
loss of the forces (e.g. force matching) come from one extra device pass.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import system, water

PARAMS = ("qH", "gamma", "sigma", "epsilon", "D", "a", "r0", "k_bend", "theta0")


def theta_of(model: water.WaterModel) -> np.ndarray:
    """Parameter vector of a TIP4P/F-like model (4 sites, M ghost)."""
    g_site, comps = next(iter(model.ghost.items()))
    gamma = dict(comps)[0]
    return np.array([model.charges[1], gamma, model.lj_sigma, model.lj_eps_kcal, model.bond["D"], model.bond["a"],
                     model.bond["r0"], model.bend_k_kcal, model.bend_theta0], dtype=np.float64)


def model_with(model: water.WaterModel, theta) -> water.WaterModel:
    """The model with parameter vector theta."""
    qH, gamma, sig, eps, D, a, r0, kb, th0 = [float(v) for v in theta]
    g_site = next(iter(model.ghost))
    return dataclasses.replace(
        model, charges=[0.0, qH, qH, -2.0 * qH], lj_sigma=sig, lj_eps_kcal=eps,
        bond={"type": "quartic", "r0": r0, "D": D, "a": a}, bend_k_kcal=kb, bend_theta0=th0,
        ghost={g_site: [(0, gamma), (1, 0.5 * (1.0 - gamma)), (2, 0.5 * (1.0 - gamma))]})


def bend_harm_coefs_dtheta0(fk, theta0):
    """d/dtheta0 (radians) of system.bend_harm_coefs: the series is a sum of
    cos(n theta0) and sin(n theta0) terms, differentiated term by term."""
    cn1, cn2, cn3, cn4 = 49.0 / 72.0, 3.0 / 4.0, 3.0 / 40.0, 1.0 / 180.0
    cn5, cn6, cn7, cn8 = 3.0 / 2.0, 3.0 / 5.0, 1.0 / 10.0, 4.0 / 15.0
    cn9, cn10, cn11 = 8.0 / 45.0, 3.0 / 10.0, 1.0 / 30.0
    # d cos(n t) = -n sin(n t), d sin(n t) = n cos(n t)
    dc2, dc4, dc6 = -2.0 * math.sin(2.0 * theta0), -4.0 * math.sin(4.0 * theta0), -6.0 * math.sin(6.0 * theta0)
    ds2, ds4, ds6 = 2.0 * math.cos(2.0 * theta0), 4.0 * math.cos(4.0 * theta0), 6.0 * math.cos(6.0 * theta0)
    c = np.array([0.5 * fk * (cn2 * dc2 + cn3 * dc4 + cn4 * dc6), 0.0,
                  0.5 * fk * (-cn5 * dc2 - cn6 * dc4 - cn7 * dc6), 0.0,
                  0.5 * fk * (cn6 * dc4 + cn8 * dc6), 0.0, 0.5 * fk * (-cn9 * dc6)])
    s = np.array([0.0, 0.0, 0.5 * fk * (-cn5 * ds2 + cn10 * ds4 - cn11 * ds6), 0.0,
                  0.5 * fk * (-cn6 * ds4 + cn9 * ds6), 0.0, 0.5 * fk * (-cn9 * ds6)])
    dc = c * np.arange(7.0)
    dc[1] = c[1]
    ds = s * np.array([0.0, 1.0, 1.0, 2.0, 3.0, 4.0, 5.0])
    return c, s, dc, ds


def tangents(spec: water.BoxSpec, theta, S: dict) -> list:
    """Derivatives of the set-up data of `system.build_system` with respect
    to each entry of theta, as pinyb200_tangent dictionaries (PARAMS order)."""
    qH, gamma, sig_A, eps_kcal, D, a, r0, kb, th0_deg = [float(v) for v in theta]
    natm, nmol = S["natm"], spec.nmol
    ns = spec.model.nsite
    BOHR, KB_KCAL, BOLTZ = water.BOHR, water.KB_KCAL, water.BOLTZ
    out = []
    # qH: charges (0, 1, 1, -2) per molecule
    out.append({"dcharge": np.tile(np.array([0.0, 1.0, 1.0, -2.0]), nmol)})
    # gamma: ghost coefficients (1, -1/2, -1/2)
    out.append({"dghost_coef": np.tile(np.array([1.0, -0.5, -0.5]), nmol)})
    # sigma, epsilon: vdW tables and the LJ tail.  For V = 4 eps ((s/r)^12 -
    # (s/r)^6), dV/ds = V(2^(1/6) s, 3 eps / s), the same switched table.
    rmin, rmax, rheal = spec.min_dist / BOHR, spec.cutoff / BOHR, 1.0 / BOHR
    sig, eps = sig_A / BOHR, (eps_kcal / KB_KCAL) / BOLTZ
    nsplin, nuniq = S["nsplin"], S["ninter_unique"]
    lj_u = None
    for u in range(nuniq):
        if np.any(S["cdv0"][u * nsplin:(u + 1) * nsplin] != 0.0):
            lj_u = u
    ds_v, ds_dv = np.zeros(nuniq * nsplin), np.zeros(nuniq * nsplin)
    de_v, de_dv = np.zeros(nuniq * nsplin), np.zeros(nuniq * nsplin)
    if lj_u is not None:
        v, dv, _, _ = system.spline_table(nsplin, rmin, rmax, "lj", 2.0 ** (1.0 / 6.0) * sig, 3.0 * eps / sig,
                                          rheal=rheal)
        ds_v[lj_u * nsplin:(lj_u + 1) * nsplin] = v / BOHR      # per Angstrom
        ds_dv[lj_u * nsplin:(lj_u + 1) * nsplin] = dv / BOHR
        v, dv, _, _ = system.spline_table(nsplin, rmin, rmax, "lj", sig, 1.0, rheal=rheal)
        deps = 1.0 / (KB_KCAL * BOLTZ)                           # Hartree per kcal/mol
        de_v[lj_u * nsplin:(lj_u + 1) * nsplin] = v * deps
        de_dv[lj_u * nsplin:(lj_u + 1) * nsplin] = dv * deps
    out.append({"dcv0": ds_v, "dcdv0": ds_dv, "dclong": 6.0 * S["clong"] / sig_A})
    out.append({"dcv0": de_v, "dcdv0": de_dv, "dclong": S["clong"] / eps_kcal})
    # bond series c2 = D a^2, c3 = -D a^3, c4 = 7/12 D a^4 (unit factors folded in)
    c = np.asarray(S["bond_c"], np.float64)
    n = np.arange(7.0)
    out.append({"dbond_c": c / D})
    out.append({"dbond_c": c * n / a})
    out.append({"dbond_eq": np.array([1.0 / BOHR])})
    # bend: series linear in k; theta0 through cos/sin(n theta0)
    fkb = (kb / KB_KCAL) / BOLTZ
    out.append({"dbend_c": np.asarray(S["bend_c"]) / kb, "dbend_s": np.asarray(S["bend_s"]) / kb,
                "dbend_dc": np.asarray(S["bend_dc"]) / kb, "dbend_ds": np.asarray(S["bend_ds"]) / kb})
    bc, bs, bdc, bds = bend_harm_coefs_dtheta0(fkb, th0_deg * math.pi / 180.0)
    f = math.pi / 180.0
    out.append({"dbend_c": bc * f, "dbend_s": bs * f, "dbend_dc": bdc * f, "dbend_ds": bds * f})
    assert natm == nmol * ns
    return out


class PinyForceField:
    """One box (positions fixed) as a function of theta on the device:
    energy (vintert + vintrat, Hartree) and forces on atoms (ghost force
    distributed) for all beads, and the adjoint through pinyb200_grad."""

    def __init__(self, spec: water.BoxSpec, pos_angstrom, precision="fp64", device="cuda:0"):
        import torch
        self.spec = spec
        self.P = spec.nbeads
        self.precision = precision
        self.device = torch.device(device)
        self.pos_bohr = np.asarray(pos_angstrom, np.float64) / water.BOHR
        self._theta = None
        self.box = None

    def _setup(self, theta):
        import torch

        from .lib import DeviceBox
        theta = np.asarray(theta, np.float64)
        if self._theta is not None and np.array_equal(theta, self._theta):
            return
        spec = dataclasses.replace(self.spec, model=model_with(self.spec.model, theta))
        S = system.build_system(spec, self.pos_bohr)
        if self.box is not None:
            self.box.close()
        self.box = DeviceBox(S, self.P, self.precision)
        xmod = self.pos_bohr.mean(axis=0) if self.P > 1 else None
        self.box.build_list(self.pos_bohr[0], xmod, S["hmat"], S["cutskin2"])
        self.box.grad_prepare(tangents(spec, theta, S))
        self.S = S
        self.hmat = S["hmat"]
        self.d_pos = torch.from_numpy(self.pos_bohr).to(self.device)
        self.d_xmod = torch.from_numpy(xmod).to(self.device) if xmod is not None else None
        self._theta = theta.copy()

    def energy_forces(self, theta):
        """(E, F[P, natm, 3]) as numpy, Hartree and Hartree/Bohr."""
        import torch
        self._setup(theta)
        f = torch.empty_like(self.d_pos)
        e = self.box.energy_force_device(self.d_pos.data_ptr(),
                                         None if self.d_xmod is None else self.d_xmod.data_ptr(),
                                         self.hmat, f.data_ptr(), distribute_ghosts=True)
        torch.cuda.synchronize()
        return e["vintert"] + e["vintrat"], f.cpu().numpy()

    def adjoint(self, theta, e_bar, f_bar):
        """e_bar dE/dtheta + sum f_bar . dF/dtheta (per PARAMS)."""
        import torch
        self._setup(theta)
        d_fbar = None
        if f_bar is not None:
            fb = torch.as_tensor(np.ascontiguousarray(f_bar, np.float64)).to(self.device)
            d_fbar = fb
        dE, dF = self.box.grad(self.d_pos.data_ptr(), None if self.d_xmod is None else self.d_xmod.data_ptr(),
                               self.hmat, None if d_fbar is None else d_fbar.data_ptr())
        torch.cuda.synchronize()
        return float(e_bar) * dE + (dF if f_bar is not None else 0.0)

    def close(self):
        if self.box is not None:
            self.box.close()
            self.box = None


def _make_function():
    import torch

    class EnergyForces(torch.autograd.Function):
        """theta (CPU float64 tensor) -> (E, F); backward runs the device
        adjoint (pinyb200_grad) once for both outputs."""

        @staticmethod
        def forward(ctx, theta, field):
            E, F = field.energy_forces(theta.detach().cpu().numpy())
            ctx.field = field
            ctx.save_for_backward(theta)
            return (torch.tensor(E, dtype=torch.float64), torch.from_numpy(F))

        @staticmethod
        def backward(ctx, e_bar, f_bar):
            (theta,) = ctx.saved_tensors
            eb = 0.0 if e_bar is None else float(e_bar)
            fb = None if f_bar is None else f_bar.detach().cpu().numpy()
            g = ctx.field.adjoint(theta.detach().cpu().numpy(), eb, fb)
            return torch.as_tensor(np.asarray(g, np.float64)), None

    return EnergyForces


_EF = None


def energy_forces(theta, field: PinyForceField):
    """Differentiable (E, F) of the box in `field` at the parameter tensor theta."""
    global _EF
    if _EF is None:
        _EF = _make_function()
    return _EF.apply(theta, field)
