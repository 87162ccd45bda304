"""PINY's NVT ring-polymer step on the device (pinyb200_pimd_forces /
pinyb200_pimd_step) against its restatement in the oracle (chains, springs,
centroid virial and transforms pinned to PINY in test_pimd_oracle.py; the
force path pinned in test_oracle_golden.py).

64 q-TIP4P/F molecules, 4 beads, staging and normal modes, FP64: mode
forces, positions, velocities and chain states agree with the oracle to
1e-11 of their scale after each of three steps; the spring energy, virial
estimator and pressure tensors to 1e-11 relative.  MIXED: mode forces
within 1e-5 (relative RMS) of FP64.  The Verlet list is built once, from
the starting positions, for both (no rebuild inside three steps)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AMU_AU = 1822.888486  # electron masses per atomic mass unit
DT = 20.0             # a.u. of time (0.48 fs)
TAU = 800.0           # chain time constant, a.u.


def _problem(kind, P=4):
    from piny_b200 import pimd, system, water
    spec = water.BoxSpec(water.TIP4P_F, 64, water.density_box_edge(64), P, 298.0, 17, grid=16, order=8)
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    natm = int(S["natm"])
    ghost = np.zeros(natm, bool)
    ghost[np.asarray(S["ghost_atom"])] = True
    mass = np.tile(np.asarray(spec.model.masses, np.float64), spec.nmol) * AMU_AU
    setup = pimd.nvt_setup(mass, ghost, P, kind, spec.temperature, DT, TAU, len_nhc=3, nres_nhc=1, nyosh=3)
    rng = np.random.default_rng(5 + kind)
    v = rng.normal(size=(P, natm, 3)) * np.sqrt(spec.temperature / water.BOLTZ / setup["bead_mass"])[:, :, None]
    v[:, ghost, :] = 0.0
    return spec, S, pos, v, setup, rng


def _chain_state(setup, rng):
    st = {}
    c, b = setup["class_nhc"], setup["bead_nhc"]
    st["cx"] = rng.normal(0, 0.05, (c["len_nhc"], c["num_nhc"]))
    st["cv"] = rng.normal(0, 1e-4, (c["len_nhc"], c["num_nhc"]))
    P = setup["nbeads"]
    st["bx"] = rng.normal(0, 0.05, (P - 1, b["len_nhc"], b["num_nhc"]))
    st["bv"] = rng.normal(0, 1e-4, (P - 1, b["len_nhc"], b["num_nhc"]))
    return st


def _close(a, b, tol):
    return np.abs(np.asarray(a) - np.asarray(b)).max() <= tol * max(1e-300, np.abs(np.asarray(b)).max())


@pytest.mark.parametrize("kind", [1, 2])
def test_device_step_matches_oracle(oracle, kind):
    import torch

    from oracle import oracle as O
    from piny_b200.lib import DeviceBox, DevicePimd
    spec, S, pos, v0, setup, rng = _problem(kind)
    P = setup["nbeads"]
    state = _chain_state(setup, rng)
    x0 = O.ghost_positions(S, pos)
    u0 = oracle.pimd_transform(x0, kind, 0)
    pi, pj = oracle.verlist(S, x0[0], u0[0], S["hmat"], S["cutskin2"])

    box = DeviceBox(S, P, "fp64")
    box.build_list(x0[0], u0[0], S["hmat"], S["cutskin2"])
    pm = DevicePimd(setup)
    pm.set_nhc(0, state["cx"], state["cv"])
    pm.set_nhc(1, state["bx"], state["bv"])
    dx = torch.from_numpy(pos.copy()).to("cuda:0")
    dv = torch.from_numpy(v0.copy()).to("cuda:0")
    df = torch.zeros_like(dx)

    ed = pm.forces(box, dx.data_ptr(), df.data_ptr(), S["hmat"])
    xo, fo, eo = O.pimd_forces(oracle, S, setup, pos, pi, pj)
    assert _close(dx.cpu().numpy(), xo, 1e-15)
    assert _close(df.cpu().numpy(), fo, 1e-11)
    assert abs(ed["kin_harm"] - eo["kin_harm"]) <= 1e-12 * abs(eo["kin_harm"])
    assert abs(ed["akvirx"] - eo["akvirx"]) <= 1e-11 * abs(eo["akvirx"])
    assert _close(ed["pvten"], eo["pvten_corr"], 1e-11)
    assert _close(ed["pvten_mode_tot"], eo["pvten_mode_tot"], 1e-12)

    x, v, f = xo, v0.copy(), fo
    for step in range(3):
        ed = pm.step(box, dx.data_ptr(), dv.data_ptr(), df.data_ptr(), S["hmat"])
        x, v, f, eo = O.pimd_step(oracle, S, setup, x, v, f, state, pi, pj)
        assert _close(dx.cpu().numpy(), x, 1e-13), step
        assert _close(dv.cpu().numpy(), v, 1e-11), step
        assert _close(df.cpu().numpy(), f, 1e-11), step
        assert abs(ed["kin_harm"] - eo["kin_harm"]) <= 1e-11 * abs(eo["kin_harm"])
        assert abs(ed["vintert"] - eo["vintert"]) <= 1e-11 * abs(eo["vintert"])
        cx, cv = pm.get_nhc(0)
        bx, bv = pm.get_nhc(1)
        assert _close(cx, state["cx"], 1e-11) and _close(cv, state["cv"], 1e-10)
        assert _close(bx, state["bx"], 1e-11) and _close(bv, state["bv"], 1e-10)
    pm.close()
    box.close()


def test_mixed_step_tracks_fp64():
    import torch

    from piny_b200.lib import DeviceBox, DevicePimd
    from oracle import oracle as O
    spec, S, pos, v0, setup, rng = _problem(2)
    P = setup["nbeads"]
    out = {}
    for prec in ("fp64", "mixed"):
        box = DeviceBox(S, P, prec)
        x0 = O.ghost_positions(S, pos)
        box.build_list(x0[0], x0.mean(axis=0), S["hmat"], S["cutskin2"])
        pm = DevicePimd(setup)
        dx = torch.from_numpy(pos.copy()).to("cuda:0")
        dv = torch.from_numpy(v0.copy()).to("cuda:0")
        df = torch.zeros_like(dx)
        pm.forces(box, dx.data_ptr(), df.data_ptr(), S["hmat"])
        pm.step(box, dx.data_ptr(), dv.data_ptr(), df.data_ptr(), S["hmat"])
        out[prec] = (df.cpu().numpy(), dx.cpu().numpy())
        pm.close()
        box.close()
    f64, f32 = out["fp64"][0], out["mixed"][0]
    assert np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()) <= 1e-5
    assert np.abs(out["mixed"][1] - out["fp64"][1]).max() <= 1e-9 * np.abs(out["fp64"][1]).max()


def test_step_arguments():
    import torch

    from piny_b200.lib import DeviceBox, DevicePimd, PinyError
    spec, S, pos, v0, setup, rng = _problem(1)
    box = DeviceBox(S, 2, "fp64")  # other bead count than the step
    pm = DevicePimd(setup)
    d = torch.zeros((4, int(S["natm"]), 3), dtype=torch.float64, device="cuda:0")
    with pytest.raises(PinyError, match="ERR_ARG"):
        pm.forces(box, d.data_ptr(), d.data_ptr(), S["hmat"])
    pm.close()
    box.close()
    bad = dict(setup)
    bad["class_nhc"] = dict(setup["class_nhc"], len_nhc=9)
    with pytest.raises(PinyError, match="ERR_ARG"):
        DevicePimd(bad)


@pytest.mark.parametrize("kind,ix_respa,nres", [(2, 1, (2, 1, 2, 1)), (1, 3, (2, 1, 2, 1)), (2, 5, (2, 1, 2, 1)),
                                               (2, 5, (1, 1, 1, 2)), (1, 4, (2, 1, 1, 2))])
def test_device_respa_step_matches_oracle(oracle, kind, ix_respa, nres):
    """int_NVT_pimd's RESPA loops on the device (inter, intra and bead
    counts as given; switch 1 Bohr below an inner cutoff 1.5 Bohr short of
    the full one, bonds' RESPA equilibrium 0.01 Bohr longer; chains at the
    level ix_respa) against the oracle's composition of the pinned pieces
    and the RESPA force split, over two outer steps."""
    import torch

    from oracle import oracle as O
    from piny_b200 import pimd, respa
    from piny_b200.lib import DeviceBox, DevicePimd
    spec, S, pos, v0, setup, rng = _problem(kind)
    P = setup["nbeads"]
    natm = int(S["natm"])
    ghost = np.zeros(natm, bool)
    ghost[np.asarray(S["ghost_atom"])] = True
    setup = pimd.nvt_setup(setup["mass"], ghost, P, kind, spec.temperature, DT * int(np.prod(nres)) / 2, TAU,
                           len_nhc=3, nres_nhc=1, nyosh=3, nres=nres, ix_respa=ix_respa)
    rs = respa.respa_setup(*nres, True, nres[0] > 1, np.asarray(S["cutoff"]) - 1.5, 1.0,
                           np.asarray(S["bond_eq"]) + 0.01)
    state = _chain_state(setup, rng)
    x0 = O.ghost_positions(S, pos)
    u0 = oracle.pimd_transform(x0, kind, 0)
    pi, pj = oracle.verlist(S, x0[0], u0[0], S["hmat"], S["cutskin2"])

    box = DeviceBox(S, P, "fp64")
    box.build_list(x0[0], u0[0], S["hmat"], S["cutskin2"])
    box.set_respa(rs)
    pm = DevicePimd(setup)
    pm.set_nhc(0, state["cx"], state["cv"])
    pm.set_nhc(1, state["bx"], state["bv"])
    dx = torch.from_numpy(pos.copy()).to("cuda:0")
    dv = torch.from_numpy(v0.copy()).to("cuda:0")
    df = torch.zeros_like(dx)
    pm.forces(box, dx.data_ptr(), df.data_ptr(), S["hmat"])
    x, f = O.pimd_forces_respa(oracle, S, setup, rs, pos, pi, pj)[:2]
    assert _close(df.cpu().numpy(), f, 1e-11)  # PINY's first call: the outer level
    v = v0.copy()
    for step in range(2):
        ed = pm.step(box, dx.data_ptr(), dv.data_ptr(), df.data_ptr(), S["hmat"])
        x, v, f, eo = O.pimd_step_respa(oracle, S, setup, rs, x, v, f, state, pi, pj)
        assert _close(dx.cpu().numpy(), x, 1e-13), step
        assert _close(dv.cpu().numpy(), v, 1e-11), step
        assert _close(df.cpu().numpy(), f, 1e-11), step
        assert abs(ed["kin_harm"] - eo["kin_harm"]) <= 1e-11 * abs(eo["kin_harm"])
        assert abs(ed["akvirx"] - eo["akvirx"]) <= 1e-10 * abs(eo["akvirx"])
        assert abs(ed["vintert"] - eo["vintert"]) <= 1e-11 * abs(eo["vintert"])
        cx, cv = pm.get_nhc(0)
        bx, bv = pm.get_nhc(1)
        assert _close(cx, state["cx"], 1e-11) and _close(cv, state["cv"], 1e-10)
        assert _close(bx, state["bx"], 1e-11) and _close(bv, state["bv"], 1e-10)
    pm.close()
    box.close()


def test_mixed_respa_step_tracks_fp64():
    """One RESPA step (counts 2, 1, 2, 1) with MIXED forces against FP64:
    mode forces within 1e-5 (relative RMS), positions within 1e-9."""
    import torch

    from oracle import oracle as O
    from piny_b200 import pimd, respa
    from piny_b200.lib import DeviceBox, DevicePimd
    spec, S, pos, v0, setup, rng = _problem(2)
    P, natm = setup["nbeads"], int(S["natm"])
    nres = (2, 1, 2, 1)
    ghost = np.zeros(natm, bool)
    ghost[np.asarray(S["ghost_atom"])] = True
    setup = pimd.nvt_setup(setup["mass"], ghost, P, 2, spec.temperature, 2 * DT, TAU, len_nhc=3, nres=nres,
                           ix_respa=5)
    rs = respa.respa_setup(*nres, True, True, np.asarray(S["cutoff"]) - 1.5, 1.0, np.asarray(S["bond_eq"]))
    out = {}
    for prec in ("fp64", "mixed"):
        box = DeviceBox(S, P, prec)
        x0 = O.ghost_positions(S, pos)
        box.build_list(x0[0], x0.mean(axis=0), S["hmat"], S["cutskin2"])
        box.set_respa(rs)
        pm = DevicePimd(setup)
        dx = torch.from_numpy(pos.copy()).to("cuda:0")
        dv = torch.from_numpy(v0.copy()).to("cuda:0")
        df = torch.zeros_like(dx)
        pm.forces(box, dx.data_ptr(), df.data_ptr(), S["hmat"])
        pm.step(box, dx.data_ptr(), dv.data_ptr(), df.data_ptr(), S["hmat"])
        out[prec] = (df.cpu().numpy(), dx.cpu().numpy())
        pm.close()
        box.close()
    f64, f32 = out["fp64"][0], out["mixed"][0]
    assert np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()) <= 1e-5
    assert np.abs(out["mixed"][1] - out["fp64"][1]).max() <= 1e-9 * np.abs(out["fp64"][1]).max()
