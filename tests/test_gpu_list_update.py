"""Device list update (pinyb200_update_list_device, PINYB200_UPDATE_LIST):
PINY's rebuild test and list build with no host round trip.

Against the oracle: the decision and cutskin^2 (bit for bit, as the host
test), the rebuilt pair set (bit-exact, sorted-pair digest) and the forces
with it (FP64, 1e-12 relative RMS); no rebuild when the displacement stays
inside half the skin; the flag path inside an evaluation and inside the
batch graph; a list that outgrows its reservation is reported (non-finite
energy, ERR_LIST_OVERFLOW) and a host build clears it."""
import numpy as np
import pytest

from helpers import load_fixture, pair_hash, rel_rms

pytestmark = pytest.mark.gpu

NAME = "tip4pf_64_p4"


def _setup(F, spread_ref=None):
    import torch

    from piny_b200.lib import DeviceBox
    P = int(F["nbeads"])
    box = DeviceBox(F, P, "fp64")
    pos = np.ascontiguousarray(F["pos"], np.float64)
    box.build_list(pos[0], F["xmod"], F["hmat"], F["cutskin2"])
    d0 = torch.from_numpy(pos).to("cuda:0")
    sp0 = box.check_list_device(d0.data_ptr(), 0.0)[2] if spread_ref is None else spread_ref
    box.list_set_spread(sp0)
    return box, pos, sp0


def _moved(pos, scale, seed):
    """Every atom moved by one random vector on all its beads: the bead
    spread stays, the displacement test sees the move."""
    rng = np.random.default_rng(seed)
    return pos + rng.normal(scale=scale, size=(1,) + pos.shape[1:])


def test_update_rebuilds_like_the_oracle(oracle):
    import torch
    F = load_fixture(NAME)
    box, pos, sp0 = _setup(F)
    skin = float(F["skin"])
    cutoff = np.asarray(F["cutoff"], np.float64)
    # small moves: no rebuild
    p1 = _moved(pos, 0.02, 1)
    d1 = torch.from_numpy(p1).to("cuda:0")
    xm1 = torch.from_numpy(np.ascontiguousarray(p1.mean(axis=0))).to("cuda:0")
    box.update_list_device(d1.data_ptr(), xm1.data_ptr(), F["hmat"])
    st = box.list_status()
    reb, rmax, sp, _ = oracle.check_list(p1, pos[0], skin, sp0, cutoff)
    assert not reb and st["rebuilt_last"] == 0 and st["rebuilds"] == 0
    assert st["rmax"] == rmax and st["spread_now"] == sp
    # large moves: rebuild on the device
    p2 = _moved(pos, 0.6, 2)
    d2 = torch.from_numpy(p2).to("cuda:0")
    x2 = p2.mean(axis=0)
    xm2 = torch.from_numpy(np.ascontiguousarray(x2)).to("cuda:0")
    box.update_list_device(d2.data_ptr(), xm2.data_ptr(), F["hmat"])
    st = box.list_status()
    reb, rmax, sp, cs = oracle.check_list(p2, pos[0], skin, sp0, cutoff)
    assert reb and st["rebuilt_last"] == 1 and st["rebuilds"] == 1
    assert st["spread_ref"] == sp
    pi, pj = oracle.verlist(F, p2[0], x2, F["hmat"], cs)
    qi, qj = box.get_list()
    assert len(qi) == len(pi) == st["npairs"]
    assert pair_hash(qi, qj) == pair_hash(pi, pj)
    df = torch.zeros_like(d2)
    e = box.energy_force_device(d2.data_ptr(), xm2.data_ptr(), F["hmat"], df.data_ptr(), distribute_ghosts=True)
    f_o, e_o = oracle.energy_force(F, p2, x2, F["hmat"], pi, pj, distribute_ghosts=True)
    assert rel_rms(df.cpu().numpy(), f_o) < 1e-12
    assert abs(e["vintert"] - e_o["vintert"]) <= 1e-11 * abs(e_o["vintert"])
    # the next test measures from the new list's positions
    box.update_list_device(d2.data_ptr(), xm2.data_ptr(), F["hmat"])
    assert box.list_status()["rebuilt_last"] == 0
    box.close()


def test_update_flag_inside_the_evaluation_and_the_graph(oracle):
    import torch

    from piny_b200.lib import DeviceBatch
    F = load_fixture(NAME)
    skin = float(F["skin"])
    cutoff = np.asarray(F["cutoff"], np.float64)
    p2 = _moved(np.ascontiguousarray(F["pos"], np.float64), 0.6, 3)
    x2 = p2.mean(axis=0)
    d2 = torch.from_numpy(p2).to("cuda:0")
    xm2 = torch.from_numpy(np.ascontiguousarray(x2)).to("cuda:0")
    for batch in (False, True):
        box, pos, sp0 = _setup(F)
        reb, _, sp, cs = oracle.check_list(p2, pos[0], skin, sp0, cutoff)
        assert reb
        pi, pj = oracle.verlist(F, p2[0], x2, F["hmat"], cs)
        f_o, e_o = oracle.energy_force(F, p2, x2, F["hmat"], pi, pj, distribute_ghosts=False)
        df = torch.zeros_like(d2)
        if batch:
            bt = DeviceBatch([box])
            for _ in range(2):  # first call captures, second replays the graph
                e = bt.energy_force_device([d2.data_ptr()], [xm2.data_ptr()], [F["hmat"]], [df.data_ptr()],
                                           update_list=True)[0]
            bt.close()
        else:
            e = box.energy_force_device(d2.data_ptr(), xm2.data_ptr(), F["hmat"], df.data_ptr(), update_list=True)
        st = box.list_status()
        assert st["rebuilds"] == 1, st
        qi, qj = box.get_list()
        assert pair_hash(qi, qj) == pair_hash(pi, pj)
        assert rel_rms(df.cpu().numpy(), f_o) < 1e-12
        assert abs(e["vintert"] - e_o["vintert"]) <= 1e-11 * abs(e_o["vintert"])
        box.close()


def test_list_that_outgrows_its_reservation_is_reported():
    import torch

    from piny_b200.lib import DeviceBox, PinyError
    F = load_fixture(NAME)
    P = int(F["nbeads"])
    pos = np.ascontiguousarray(F["pos"], np.float64)
    box = DeviceBox(F, P, "fp64")
    # a host list of very short reach reserves little room ...
    box.build_list(pos[0], F["xmod"], F["hmat"], np.full_like(np.asarray(F["cutskin2"]), 4.0))
    small = box.list_info()["npairs"]
    d0 = torch.from_numpy(pos).to("cuda:0")
    box.list_set_spread(box.check_list_device(d0.data_ptr(), 0.0)[2])
    # ... and the device rebuild at full reach does not fit
    p2 = _moved(pos, 0.6, 4)
    d2 = torch.from_numpy(p2).to("cuda:0")
    xm2 = torch.from_numpy(np.ascontiguousarray(p2.mean(axis=0))).to("cuda:0")
    box.update_list_device(d2.data_ptr(), xm2.data_ptr(), F["hmat"])
    with pytest.raises(PinyError, match="ERR_LIST_OVERFLOW"):
        box.list_status()
    df = torch.zeros_like(d2)
    with pytest.raises(PinyError, match="ERR_NAN"):
        box.energy_force_device(d2.data_ptr(), xm2.data_ptr(), F["hmat"], df.data_ptr())
    # a host build at full reach grows the reservation and clears the state
    box.build_list(p2[0], p2.mean(axis=0), F["hmat"], F["cutskin2"])
    assert box.list_info()["npairs"] > small
    box.list_status()
    box.energy_force_device(d2.data_ptr(), xm2.data_ptr(), F["hmat"], df.data_ptr())
    box.close()


def test_update_arguments_and_state():
    import torch

    from piny_b200.lib import DeviceBox, PinyError
    F = load_fixture(NAME)
    P = int(F["nbeads"])
    box = DeviceBox(F, P, "fp64")
    d = torch.from_numpy(np.ascontiguousarray(F["pos"], np.float64)).to("cuda:0")
    xm = torch.from_numpy(np.ascontiguousarray(F["xmod"], np.float64)).to("cuda:0")
    with pytest.raises(PinyError, match="ERR_STATE"):  # no host build yet
        box.update_list_device(d.data_ptr(), xm.data_ptr(), F["hmat"])
    box.build_list(F["pos"][0], F["xmod"], F["hmat"], F["cutskin2"])
    with pytest.raises(PinyError, match="ERR_ARG"):  # beads without mode-1 positions
        box.update_list_device(d.data_ptr(), None, F["hmat"])
    st = box.list_status()
    assert st["rebuilds"] == 0 and st["overflow"] == 0 and st["npairs"] == box.list_info()["npairs"]
    box.close()
