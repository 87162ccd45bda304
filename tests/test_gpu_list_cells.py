"""Link-cell list build (PINYB200_LIST_LNK, PINY's lnk_ver_update) against
the all-pairs sweep (PINYB200_LIST_NOLST, nolst_ver_update) and the oracle.

The pair sets must be identical bit for bit (sorted-pair digest): at 32768
molecules against the sweep over the whole list and against the oracle on
sampled rows; in a sheared cell against the sweep and the oracle's rows
(and, with the sweep, against the oracle over a whole smaller list); for
a device rebuild with the host build's cell plan; and when the molecules'
reach outgrows that plan, which must send the device rebuild to the sweep.
Forces and energies with the two lists agree to summation order (FP64)."""
import numpy as np
import pytest

from helpers import pair_hash, rel_rms

pytestmark = pytest.mark.gpu


def _box(model, nmol, nbeads, seed, shear=None):
    from piny_b200 import system, water
    spec = water.BoxSpec(model, nmol, water.density_box_edge(nmol), nbeads, 298.0, seed, grid=32, order=6)
    pos = water.build_positions(spec) / water.BOHR
    h = None
    if shear is not None:
        L = spec.L / water.BOHR
        h = np.array([L, 0.0, 0.0, shear[0] * L, L, 0.0, shear[1] * L, shear[2] * L, L])
    S = system.build_system(spec, pos, hmat=h)
    return spec, pos, S


def _list(box, method, pos1, xmod, S, cs=None):
    from piny_b200 import lib
    box.set_list_method(method)
    n = box.build_list(pos1, xmod, S["hmat"], S["cutskin2"] if cs is None else cs)
    pi, pj = box.get_list()
    assert n == len(pi)
    return pi, pj, box.list_cells()


def test_cells_match_the_sweep_and_the_oracle_at_32k_molecules(oracle):
    from piny_b200 import lib, water
    from piny_b200.lib import DeviceBox
    spec, pos, S = _box(water.TIP4P_F, 32768, 4, 7)
    xmod = pos.mean(axis=0)
    box = DeviceBox(S, spec.nbeads, "fp64")
    ci, cj, (cells, used) = _list(box, lib.LIST_LNK, pos[0], xmod, S)
    assert min(cells) >= 5 and used, cells
    f_c, e_c = box.energy_force(pos, xmod, S["hmat"])
    si, sj, (cells_s, used_s) = _list(box, lib.LIST_NOLST, pos[0], xmod, S)
    assert cells_s == (0, 0, 0) and not used_s
    assert len(ci) == len(si) and pair_hash(ci, cj) == pair_hash(si, sj)
    f_s, e_s = box.energy_force(pos, xmod, S["hmat"])
    assert rel_rms(f_c, f_s) < 1e-13
    assert abs(e_c["vintert"] - e_s["vintert"]) <= 1e-12 * abs(e_s["vintert"])
    # the oracle on rows across the box (site rows of 64 molecules each)
    ns = water.TIP4P_F.nsite
    for m0 in (0, 9000, 20011, 32704):
        ilo, ihi = ns * m0, ns * (m0 + 64)
        oi, oj = oracle.verlist_rows(S, pos[0], xmod, S["hmat"], S["cutskin2"], ilo, ihi)
        sel = (ci >= ilo) & (ci < ihi)
        assert len(oi) > 0 and pair_hash(ci[sel], cj[sel]) == pair_hash(oi, oj)
    box.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_cells_in_a_sheared_cell_match_the_sweep_and_the_oracle(prec, oracle):
    from piny_b200 import lib, water
    from piny_b200.lib import DeviceBox
    spec, pos, S = _box(water.SPC_FW, 12000, 2, 11, shear=(0.12, -0.07, 0.05))
    xmod = pos.mean(axis=0)
    box = DeviceBox(S, spec.nbeads, prec)
    ci, cj, (cells, used) = _list(box, lib.LIST_LNK, pos[0], xmod, S)
    assert min(cells) >= 5 and used, cells
    si, sj, _ = _list(box, lib.LIST_NOLST, pos[0], xmod, S)
    assert len(ci) == len(si) and pair_hash(ci, cj) == pair_hash(si, sj)
    ns = water.SPC_FW.nsite
    for m0 in (0, 5003, 11936):
        ilo, ihi = ns * m0, ns * (m0 + 64)
        oi, oj = oracle.verlist_rows(S, pos[0], xmod, S["hmat"], S["cutskin2"], ilo, ihi)
        sel = (ci >= ilo) & (ci < ihi)
        assert len(oi) > 0 and pair_hash(ci[sel], cj[sel]) == pair_hash(oi, oj)
    box.close()


def test_sweep_in_a_sheared_cell_matches_the_oracle(oracle):
    """A sheared box too small for cells: the sweep over the whole list."""
    from piny_b200 import lib, water
    from piny_b200.lib import DeviceBox
    spec, pos, S = _box(water.SPC_FW, 3000, 2, 12, shear=(0.12, -0.07, 0.05))
    xmod = pos.mean(axis=0)
    box = DeviceBox(S, spec.nbeads, "fp64")
    ci, cj, (cells, used) = _list(box, lib.LIST_LNK, pos[0], xmod, S)
    assert cells == (0, 0, 0) and not used
    oi, oj = oracle.verlist(S, pos[0], xmod, S["hmat"], S["cutskin2"])
    assert len(ci) == len(oi) and pair_hash(ci, cj) == pair_hash(oi, oj)
    box.close()


def _moved(pos, scale, seed):
    rng = np.random.default_rng(seed)
    return pos + rng.normal(scale=scale, size=(1,) + pos.shape[1:])


def _device_rebuild(oracle, spec, pos, S, p2):
    """Host build with cells at pos, device rebuild at p2; the device list,
    whether the cells built it, and the oracle's cutskin^2 for p2."""
    import torch

    from piny_b200 import lib
    from piny_b200.lib import DeviceBox
    box = DeviceBox(S, spec.nbeads, "fp64")
    _list(box, lib.LIST_LNK, pos[0], pos.mean(axis=0), S)
    d0 = torch.from_numpy(pos).to("cuda:0")
    sp0 = box.check_list_device(d0.data_ptr(), 0.0)[2]
    box.list_set_spread(sp0)
    d2 = torch.from_numpy(p2).to("cuda:0")
    xm2 = torch.from_numpy(np.ascontiguousarray(p2.mean(axis=0))).to("cuda:0")
    box.update_list_device(d2.data_ptr(), xm2.data_ptr(), S["hmat"])
    st = box.list_status()
    reb, _, _, cs = oracle.check_list(p2, pos[0], float(S["skin"]), sp0, np.asarray(S["cutoff"], np.float64))
    assert reb and st["rebuilt_last"] == 1
    qi, qj = box.get_list()
    cells = box.list_cells()
    # the sweep at p2 with the device's cutskin^2, from a second context
    ref = DeviceBox(S, spec.nbeads, "fp64")
    si, sj, _ = _list(ref, lib.LIST_NOLST, p2[0], p2.mean(axis=0), S, cs=cs)
    ref.close()
    box.close()
    return qi, qj, cells, si, sj


def test_device_rebuild_with_cells_matches_the_sweep(oracle):
    from piny_b200 import water
    spec, pos, S = _box(water.TIP4P_F, 8000, 4, 5)
    p2 = _moved(pos, 0.6, 2)
    qi, qj, (cells, used), si, sj = _device_rebuild(oracle, spec, pos, S, p2)
    assert min(cells) >= 5 and used
    assert len(qi) == len(si) and pair_hash(qi, qj) == pair_hash(si, sj)


@pytest.mark.parametrize("case", ["stretch", "pile"])
def test_device_rebuild_beyond_the_cell_plan_sweeps(case, oracle):
    """stretch: ten molecules stretched to four times their size about site
    0 (every bead's offset from its centroid kept, so the bead spread and
    cutskin stay) give a reach of 39 Bohr, past the 33.5 Bohr the host
    build's 7 x 7 x 7 cells were planned for.  pile: 300 molecules moved
    onto one point overfill a cell."""
    from piny_b200 import water
    spec, pos, S = _box(water.TIP4P_F, 8000, 4, 5)
    cen = pos.mean(axis=0)
    ns = water.TIP4P_F.nsite
    c = cen.reshape(-1, ns, 3).copy()
    if case == "stretch":
        c[:10] = c[:10, :1] + 4.0 * (c[:10] - c[:10, :1])
    else:
        rng = np.random.default_rng(4)
        k = rng.choice(len(c), 300, replace=False)
        c[k] += (c[k[0], 0] - c[k, 0])[:, None, :] + rng.uniform(-0.05, 0.05, size=(300, 1, 3))
    p2 = c.reshape(-1, 3)[None] + (pos - cen)
    qi, qj, (cells, used), si, sj = _device_rebuild(oracle, spec, pos, S, p2)
    assert min(cells) >= 5 and not used
    assert len(qi) == len(si) and pair_hash(qi, qj) == pair_hash(si, sj)
