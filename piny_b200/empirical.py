"""PINY's Python interface over the device path.

`PINYEmpirical` keeps the interface of PINY's Cython class of the same name
(python/piny/piny.pyx:15-436): P replicas of one empirical force-field
set-up, each parsed from its own PINY input directory, with get_n_atoms,
get_P, get_m, get_names, get_hmat, get_pbc, get_charges, get_x / set_x
(positions as n_atoms x 3 x P, ghost positions recomputed as
get_ghost_pos does), update (one force evaluation of every replica),
get_V (vintert + vintrat per replica, piny.pyx:367-384) and get_dV_dx
(minus the forces, piny.pyx:386-424).  PINY evaluates the replicas with
energy_control from OpenMP threads (piny.pyx:426-436); here they are
independent boxes of one pinyb200 batch -- one CUDA graph launch per update
-- and each keeps its own Verlet list, tested and rebuilt on the device
exactly when PINY's nbr_list_control would (PINY builds the first list while
parsing, so the constructor does).

The set-up comes from this package: the input directory is read
(`read_water_input`: PINY's input language for the flexible point-charge
water models this path serves -- the main input, the molecule set, the
.parm, .bond, .bend and .inter files and the .initial start file) and
`piny_b200.system.build_system` restates PINY's set-up from it.

`CalculatorPINY` / `atoms_from_PINY` follow python/piny/ase.py:12-89 (ASE
energy and forces in eV and eV/Angstrom); `energy_forces` is the
differentiable entry point (`piny_b200.params.energy_forces`) for the
q-TIP4P/F parameter vector of one replica.
"""
from __future__ import annotations

import os
import re
import shutil

import numpy as np

from . import files, system, water

MASS_AU = 1822.888486  # electron masses per amu (PINY's mass unit)


# ---------------------------------------------------------------------------
# PINY input language (the subset the water models use)

def read_sections(path):
    """[(section, {key: value})] of a PINY input file: ~name[ \\key{value} ... ]."""
    with open(path) as f:
        text = f.read()
    out = []
    for m in re.finditer(r"~(\w+)\[(.*?)\]", text, re.S):
        keys = {k: v.strip() for k, v in re.findall(r"\\(\w+)\{([^}]*)\}", m.group(2))}
        out.append((m.group(1), keys))
    return out


def _one(sections, name):
    for n, d in sections:
        if n == name:
            return d
    return {}


def read_water_input(directory, fn_input):
    """(BoxSpec, positions [P][natm][3] in Bohr) of a PINY input directory
    for a flexible point-charge water model (q-SPC/Fw-like 3 sites, or
    q-TIP4P/F-like 4 sites with an M ghost), as PINY reads it: energies in
    K, lengths in Angstrom, the power-series or harmonic OH bond, the
    harmonic HOH bend, Lennard-Jones between O sites only."""
    main = read_sections(os.path.join(directory, fn_input))
    gen = _one(main, "sim_gen_def")
    pimd = _one(main, "sim_pimd_def")
    lst = _one(main, "sim_list_def")
    pe = _one(main, "sim_class_PE_def")
    wr = _one(main, "sim_write_def")
    if pe.get("shift_inter_pe", "swit") != "swit":
        raise ValueError("shift_inter_pe %s: only the switched tables are supported" % pe.get("shift_inter_pe"))
    if pe.get("ewald_pme_opt", "on") != "on":
        raise ValueError("ewald_pme_opt off: the device path computes the reciprocal sum by PME")
    nbeads = int(pimd.get("path_int_beads", 1))
    mset = read_sections(os.path.join(directory, wr["mol_set_file"]))
    mdef = _one(mset, "molecule_def")
    db = _one(mset, "data_base_def")
    parm = read_sections(os.path.join(directory, mdef["mol_parm_file"]))
    atoms = sorted([d for n, d in parm if n == "atom_def"], key=lambda d: int(d["atom_ind"]))
    sites = [d["atom_typ"] for d in atoms]
    ghost = {}
    for i, d in enumerate(atoms):
        comps = []
        for c in range(1, 10):
            v = d.get("def_ghost%d" % c)
            if v is None:
                break
            j, coef = v.split(",")
            comps.append((int(j) - 1, float(coef)))
        if comps:
            ghost[i] = comps
    bond = _one(read_sections(os.path.join(directory, db["bond_file"])), "bond_parm")
    if bond["pot_type"] == "harm":
        bmodel = {"type": "harm", "r0": float(bond["eq"]), "k": float(bond["fk"]) * water.KB_KCAL}
    elif bond["pot_type"] == "power":
        p2, p3 = float(bond["p2"]), float(bond["p3"])
        a = -p3 / p2
        bmodel = {"type": "quartic", "r0": float(bond["eq"]), "D": p2 / (a * a) * water.KB_KCAL, "a": a}
    else:
        raise ValueError("bond pot_type %s is not one of harm, power" % bond["pot_type"])
    bend = _one(read_sections(os.path.join(directory, db["bend_file"])), "bend_parm")
    inter = [d for n, d in read_sections(os.path.join(directory, db["inter_file"])) if n == "inter_parm"]
    sig = eps = 0.0
    cut = mind = None
    for d in inter:
        if d["pot_type"] == "lennard-jones":
            sig, eps = float(d["sig"]), float(d["eps"]) * water.KB_KCAL
        cut = float(d["max_dist"]) if cut is None else cut
        mind = float(d.get("min_dist", 0.1)) if mind is None else mind
    model = water.WaterModel(
        name="input", sites=sites, masses=[float(d["mass"]) for d in atoms],
        charges=[float(d["charge"]) for d in atoms], lj_sigma=sig, lj_eps_kcal=eps, bond=bmodel,
        bend_theta0=float(bend["eq_bend"]), bend_k_kcal=float(bend["fk_bend"]) * water.KB_KCAL, ghost=ghost)
    nmol = int(mdef["num_mol"])
    pos, cell, _ = files.read_initial(os.path.join(directory, wr["in_restart_file"]), natm=nmol * len(sites))
    L = float(cell[0][0])
    spec = water.BoxSpec(model, nmol, L, nbeads=nbeads, temperature=float(gen.get("temperature", 300.0)), seed=0,
                         cutoff=cut, min_dist=mind, skin=float(lst.get("verlist_skin", 1.0)),
                         alpha=float(pe["ewald_alpha"]) / L, order=int(pe["ewald_interp_pme"]),
                         kmax=int(pe["ewald_kmax"]), nsplin=int(pe.get("inter_spline_pts", 2000)),
                         kmax_pme_in=int(pe["ewald_kmax_pme"]))
    return spec, pos


# ---------------------------------------------------------------------------

class PINYEmpirical:
    """P replicas of one empirical force-field set-up (python/piny/piny.pyx:15).

    template_dir_work: the work directory, or with P > 1 a %-template of one
    per replica (``template_dir_work % i``); dir_source: copied to each work
    directory first when given; fn_input: the PINY input file there; fn_out:
    a log file written in each work directory (PINY's set-up output goes
    there in the original).  precision: "fp64" (PINY's arithmetic) or
    "mixed"."""

    def __init__(self, template_dir_work, fn_input, fn_out, dir_source=None, P=1, precision="fp64",
                 device="cuda:0"):
        import torch

        from .lib import DeviceBatch, DeviceBox

        dirs = [template_dir_work] if P == 1 else [template_dir_work % i for i in range(P)]
        self._P = P
        self._boxes, self._S, self._specs = [], [], []
        self._x = None
        self._dev = torch.device(device)
        xs = []
        for d in dirs:
            if dir_source is not None:
                if os.path.isdir(d):
                    shutil.rmtree(d)
                shutil.copytree(dir_source, d)
            spec, pos = read_water_input(d, fn_input)
            if spec.nbeads != 1 or pos.shape[0] != 1:
                raise ValueError("%s: path-integral input; PINYEmpirical replicas are classical" % d)
            S = system.build_system(spec, pos)
            box = DeviceBox(S, 1, precision)
            box.build_list(pos[0], None, S["hmat"], S["cutskin2"])  # PINY's list of the parse step
            with open(os.path.join(d, fn_out), "w") as f:
                f.write("pinyb200: %d atoms, %d pairs in the Verlet list, PME %dx%dx%d order %d, %s\n"
                        % (S["natm"], box.list_info()["npairs"], S["ngrid_a"], S["ngrid_b"], S["ngrid_c"],
                           S["n_interp"], precision))
            self._boxes.append(box)
            self._S.append(S)
            self._specs.append(spec)
            xs.append(pos[0])
        self._n_atoms = int(self._S[0]["natm"])
        if any(int(S["natm"]) != self._n_atoms for S in self._S):
            raise ValueError("replicas differ in their number of atoms")
        self._x = np.stack(xs, axis=2)  # n_atoms x 3 x P, Bohr
        self._f = np.zeros_like(self._x)
        self._V = np.zeros(P)
        self._batch = DeviceBatch(self._boxes)
        n = self._n_atoms
        self._d_pos = [torch.zeros((1, n, 3), dtype=torch.float64, device=self._dev) for _ in range(P)]
        self._d_f = [torch.zeros((1, n, 3), dtype=torch.float64, device=self._dev) for _ in range(P)]
        self._pin = torch.zeros((P, n, 3), dtype=torch.float64).pin_memory()
        self._pin_f = torch.zeros((P, n, 3), dtype=torch.float64).pin_memory()
        self._fields = {}

    # -- queries (piny.pyx:200-327) ------------------------------------------
    def get_n_atoms(self):
        return self._n_atoms

    def get_P(self):
        return self._P

    def get_m(self):
        """Atomic masses (electron masses), from the first replica."""
        m = self._specs[0].model
        return np.tile(np.asarray(m.masses, np.float64), self._specs[0].nmol) * MASS_AU

    def get_names(self):
        m = self._specs[0].model
        return list(m.sites) * self._specs[0].nmol

    def get_hmat(self):
        """Cell with the box vectors in columns (Bohr)."""
        return np.asarray(self._S[0]["hmat"], np.float64).reshape(3, 3, order="F")

    def get_pbc(self):
        return [True, True, True]

    def get_charges(self):
        return np.asarray(self._S[0]["charge"], np.float64).copy()

    def get_x(self):
        """Positions of all replicas, n_atoms x 3 x P (Bohr)."""
        return self._x.copy()

    def set_x(self, x):
        """Positions from an n_atoms x 3 x P array; ghost sites (the M site)
        recomputed from their components as get_ghost_pos does
        (ghost_control.c:28-69)."""
        x = np.array(x, np.float64).reshape(self._n_atoms, 3, self._P)
        S = self._S[0]
        ng = int(S.get("nghost", 0))
        if ng:
            nc = int(S["ghost_ncomp"])
            comp = np.asarray(S["ghost_comp"]).reshape(ng, nc)
            coef = np.asarray(S["ghost_coef"]).reshape(ng, nc)
            g = np.asarray(S["ghost_atom"])
            acc = np.zeros((ng, 3, self._P))
            for c in range(nc):
                ok = comp[:, c] >= 0
                acc[ok] += coef[ok, c][:, None, None] * x[comp[ok, c]]
            x[g] = acc
        self._x = x

    # -- evaluation (piny.pyx:426-436) ---------------------------------------
    def update(self):
        """One evaluation of forces and potential energy of every replica,
        after PINY's list test (and rebuild where it fires) per replica."""
        import torch
        self._pin.copy_(torch.from_numpy(np.ascontiguousarray(np.moveaxis(self._x, 2, 0))))
        stream = torch.cuda.current_stream(self._dev)
        for i in range(self._P):
            self._d_pos[i][0].copy_(self._pin[i], non_blocking=True)
        es = self._batch.energy_force_device([d.data_ptr() for d in self._d_pos], [None] * self._P,
                                             [S["hmat"] for S in self._S], [f.data_ptr() for f in self._d_f],
                                             stream=stream.cuda_stream, update_list=True)
        for i in range(self._P):
            self._pin_f[i].copy_(self._d_f[i][0], non_blocking=True)
        torch.cuda.synchronize(self._dev)
        self._f = np.moveaxis(self._pin_f.numpy(), 0, 2).copy()
        self._V = np.array([e["vintert"] + e["vintrat"] for e in es])

    def get_V(self, V=None):
        """Potential energy (Hartree) of each replica at the last update."""
        if V is None:
            V = np.empty(self._P)
        V[:] = self._V
        return V

    def get_dV_dx(self, dV_dx=None):
        """Energy derivatives (minus the forces, Hartree/Bohr), n_atoms x 3 x P,
        at the last update (ghost forces left on the ghosts, as PINY's
        energy_control leaves them for energy_control_final)."""
        if dV_dx is None:
            dV_dx = np.empty((self._n_atoms, 3, self._P))
        dV_dx[:] = -self._f
        return dV_dx

    def list_rebuilds(self):
        """Device list builds per replica since construction (PINY's
        stat_avg.updates)."""
        return [b.list_status()["rebuilds"] for b in self._boxes]

    # -- parameters --------------------------------------------------------
    def energy_forces(self, theta, replica=0, precision=None):
        """Differentiable (E, F) of one replica at the q-TIP4P/F parameter
        tensor theta (piny_b200.params.PARAMS), forces on atoms with the
        ghost forces distributed; backward is the device adjoint."""
        from . import params
        key = (replica, precision)
        if key not in self._fields:
            spec = self._specs[replica]
            self._fields[key] = params.PinyForceField(
                spec, np.moveaxis(self._x[:, :, replica:replica + 1], 2, 0) * water.BOHR,
                precision or self._boxes[replica].precision, device=str(self._dev))
        return params.energy_forces(theta, self._fields[key])

    def close(self):
        for f in self._fields.values():
            f.close()
        self._fields = {}
        if getattr(self, "_batch", None) is not None:
            self._batch.close()
            self._batch = None
        for b in getattr(self, "_boxes", []):
            b.close()
        self._boxes = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# ASE (python/piny/ase.py:12-89)

BOHR_A = water.BOHR
HARTREE_EV = 27.211386245988


def _calculator_base():
    try:
        from ase.calculators.calculator import Calculator
        return Calculator
    except ImportError:
        class Calculator:
            """The part of ase.calculators.calculator.Calculator this
            calculator uses, for hosts without ASE."""
            implemented_properties = []

            def __init__(self):
                self.results = {}
                self.atoms = None

            def calculate(self, atoms=None, properties=("energy",), system_changes=None):
                if atoms is not None:
                    self.atoms = atoms

            def get_potential_energy(self, atoms=None):
                self.calculate(atoms if atoms is not None else self.atoms, ["energy"], {"positions"})
                return self.results["energy"]

            def get_forces(self, atoms=None):
                self.calculate(atoms if atoms is not None else self.atoms, ["forces"], {"positions"})
                return self.results["forces"]
        return Calculator


class CalculatorPINY(_calculator_base()):
    """Energy (eV) and forces (eV/Angstrom) of a one-replica PINYEmpirical."""

    implemented_properties = ["energy", "forces"]
    changes = {"positions"}

    def __init__(self, sim):
        super().__init__()
        self.sim = sim
        self.results = {}

    def calculate(self, atoms=None, properties=("energy",), system_changes=("positions",)):
        sim = self.sim
        if system_changes is not None and not self.changes.issuperset(system_changes):
            raise NotImplementedError("Not all changes are supported: %s" % (system_changes,))
        # positions to the device path, ghosts recomputed and set back
        sim.set_x((atoms.get_positions() / BOHR_A)[:, :, np.newaxis])
        atoms.set_positions(sim.get_x()[:, :, 0] * BOHR_A)
        super().calculate(atoms=atoms)
        sim.update()
        self.results = {"energy": float(sim.get_V()[0]) * HARTREE_EV,
                        "forces": -sim.get_dV_dx()[:, :, 0] * HARTREE_EV / BOHR_A}


def atoms_from_PINY(sim, types2elements=None):
    """An ase.Atoms of the first replica with a CalculatorPINY attached."""
    from ase.atoms import Atoms
    names = sim.get_names()
    if types2elements is not None:
        names = [types2elements.get(n, n) for n in names]
    atoms = Atoms(symbols=names, positions=sim.get_x()[:, :, 0] * BOHR_A, masses=sim.get_m() / MASS_AU,
                  cell=sim.get_hmat().T * BOHR_A, pbc=sim.get_pbc(), charges=sim.get_charges())
    calc = CalculatorPINY(sim)
    atoms.calc = calc
    calc.atoms = atoms
    return atoms
