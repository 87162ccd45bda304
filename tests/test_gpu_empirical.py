"""PINYEmpirical over the device path: the calling sequence of PINY's
python/piny interface (set_x, update, get_V, get_dV_dx; the ASE calculator;
the differentiable parameter call) against PINY itself and the oracle.

Tolerances: FP64, forces relative RMS 1e-12, energies 1e-11 relative.
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import read_piny_dump, rel_rms

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF = os.path.join(ROOT, "oracle", "_ref", "piny_ref")


def _replicas(tmp_path, P=2):
    from piny_b200 import water
    spec = water.BoxSpec(water.TIP4P_F, 64, 12.416, 1, 298.0, 0, cutoff=6.0, grid=16, order=8, kmax=6)
    import dataclasses
    dirs = []
    for i in range(P):
        sp = dataclasses.replace(spec, seed=200 + i)
        d = str(tmp_path / ("rep%d" % i))
        water.write_piny_input(d, sp, water.build_positions(sp))
        dirs.append(d)
    return str(tmp_path / "rep%d"), dirs


def test_empirical_sequence_matches_piny_and_oracle(tmp_path, oracle):
    from piny_b200 import empirical, system
    template, dirs = _replicas(tmp_path)
    sim = empirical.PINYEmpirical(template, "water.input", "pinyb200.log", P=2)
    assert sim.get_P() == 2 and sim.get_n_atoms() == 256
    assert sim.get_names()[:4] == ["O", "H", "H", "M"]
    assert sim.get_m()[0] == pytest.approx(15.999 * 1822.888486)
    x = sim.get_x()
    assert x.shape == (256, 3, 2)
    sim.update()
    V, G = sim.get_V(), sim.get_dV_dx()
    # PINY itself on each replica's input (copied: PINY writes its outputs there)
    if os.path.exists(REF):
        for i, d in enumerate(dirs):
            dc = str(tmp_path / ("piny%d" % i))
            subprocess.run(["cp", "-r", d, dc], check=True)
            out = str(tmp_path / ("piny%d.bin" % i))
            subprocess.run([REF, "dump", dc, "water.input", out], check=True, capture_output=True)
            D = read_piny_dump(out)
            f = D["force_raw"].reshape(-1, 3)
            assert rel_rms(-G[:, :, i], f) < 1e-12
            vref = float(D["vintert"][0] + D["vintrat"][0])
            assert abs(V[i] - vref) <= 1e-11 * abs(vref)
    # moved positions: a small move keeps each replica's list, a large one
    # rebuilds it (PINY's list test, per replica)
    rng = np.random.default_rng(5)
    for scale, rebuilt in ((0.02, False), (0.6, True)):
        before = sim.list_rebuilds()
        x2 = x + rng.normal(scale=scale, size=x.shape)
        sim.set_x(x2)
        x2 = sim.get_x()  # ghosts recomputed from the moved O, H, H
        sim.update()
        after = sim.list_rebuilds()
        assert [a > b for a, b in zip(after, before)] == [rebuilt, rebuilt]
        for i in range(2):
            S = sim._S[i]
            pos = np.ascontiguousarray(x2[:, :, i])[None]
            ref_pos = pos[0] if rebuilt else x[:, :, i]
            pi, pj = oracle.verlist(S, ref_pos, None, S["hmat"], S["cutskin2"])
            fref, eref = oracle.energy_force(S, pos, None, S["hmat"], pi, pj)
            assert rel_rms(-sim.get_dV_dx()[:, :, i], fref[0]) < 1e-12
            vref = eref["vintert"] + eref["vintrat"]
            assert abs(sim.get_V()[i] - vref) <= 1e-11 * abs(vref)
        x = x2 if rebuilt else x
    sim.close()


def test_ase_calculator_and_parameter_gradient(tmp_path):
    import torch

    from piny_b200 import empirical, params
    template, dirs = _replicas(tmp_path, P=1)
    sim = empirical.PINYEmpirical(dirs[0], "water.input", "pinyb200.log", P=1)

    class Atoms:  # the two methods the calculator uses
        def __init__(self, p):
            self.p = p

        def get_positions(self):
            return self.p.copy()

        def set_positions(self, p):
            self.p = np.asarray(p).copy()

    atoms = Atoms(sim.get_x()[:, :, 0] * empirical.BOHR_A)
    calc = empirical.CalculatorPINY(sim)
    calc.calculate(atoms, ["energy", "forces"], ["positions"])
    e_ev, f_ev = calc.results["energy"], calc.results["forces"]
    assert e_ev == pytest.approx(sim.get_V()[0] * empirical.HARTREE_EV, rel=1e-14)
    assert np.allclose(f_ev, -sim.get_dV_dx()[:, :, 0] * empirical.HARTREE_EV / empirical.BOHR_A, rtol=0, atol=0)
    with pytest.raises(NotImplementedError):
        calc.calculate(atoms, ["energy"], ["cell"])
    # differentiable call at the model's own parameters: the same energy;
    # backward gives dE/dtheta from the device adjoint
    theta = torch.tensor(params.theta_of(sim._specs[0].model), dtype=torch.float64, requires_grad=True)
    E, F = sim.energy_forces(theta)
    assert float(E.detach()) == pytest.approx(sim.get_V()[0], rel=1e-11)
    E.backward()
    assert theta.grad is not None and torch.all(torch.isfinite(theta.grad))
    sim.close()
