"""pinyb200_count_list_device: the allocation-free pair count.

Compared, call after call, with the list pinyb200_build_list builds for the
same positions (pair counts are integers: the tolerance is zero).  The file
is named to be collected last so that it also runs after every other test in
the same process; it passes alone as well.
"""
import dataclasses

import numpy as np
import pytest

from helpers import load_fixture

pytestmark = pytest.mark.gpu


def _counts_from_build_list(box, pos1, xmod, hmat, cutskin2):
    n = box.build_list(pos1, xmod, hmat, cutskin2)
    info = box.list_info()
    assert info["npairs"] == n
    return n, info["nactive"]


@pytest.mark.parametrize("name", ["tip4pf_64_p4", "spcfw_64_p1"])
def test_count_matches_build_list_on_consecutive_calls(name):
    import torch

    from piny_b200.lib import DeviceBox

    F = load_fixture(name)
    box = DeviceBox(F, int(F["nbeads"]), "fp64")
    xmod = F.get("xmod")
    hmat, cs = F["hmat"], F["cutskin2"]
    pos_a = np.ascontiguousarray(F["pos"][0], np.float64)
    rng = np.random.default_rng(7)
    pos_b = pos_a + rng.normal(scale=0.4, size=pos_a.shape)  # Bohr; changes the pair set

    dev = torch.device("cuda:0")
    d_a = torch.from_numpy(pos_a).to(dev)
    d_b = torch.from_numpy(pos_b).to(dev)
    d_xm = None if xmod is None else torch.from_numpy(np.ascontiguousarray(xmod, np.float64)).to(dev)
    xm_ptr = None if d_xm is None else d_xm.data_ptr()
    torch.cuda.synchronize()

    ref_a = _counts_from_build_list(box, pos_a, xmod, hmat, cs)
    ref_b = _counts_from_build_list(box, pos_b, xmod, hmat, cs)
    assert ref_a != ref_b

    # consecutive calls: the totals must be cleared between them
    assert box.count_list_device(d_a.data_ptr(), xm_ptr, hmat, cs) == ref_a
    assert box.count_list_device(d_a.data_ptr(), xm_ptr, hmat, cs) == ref_a
    assert box.count_list_device(d_b.data_ptr(), xm_ptr, hmat, cs) == ref_b
    assert box.count_list_device(d_a.data_ptr(), xm_ptr, hmat, cs) == ref_a

    # on a caller's stream
    s = torch.cuda.Stream()
    assert box.count_list_device(d_b.data_ptr(), xm_ptr, hmat, cs, stream=s.cuda_stream) == ref_b
    assert box.count_list_device(d_b.data_ptr(), xm_ptr, hmat, cs, stream=s.cuda_stream) == ref_b

    # the context's own list is untouched by the count
    assert box.list_info()["npairs"] == ref_b[0]
    box.close()


def test_count_rejects_sizes_beyond_the_scratch():
    import torch

    from piny_b200 import system, water
    from piny_b200.lib import COUNT_MAX_ATOMS, DeviceBox, PinyError

    base = water.named_spec("spcfw_256_p1")
    nmol = COUNT_MAX_ATOMS // 3 + 1
    spec = dataclasses.replace(base, nmol=nmol, L=(nmol * 29.92) ** (1.0 / 3.0), grid=16, kmax=0)
    pos = water.build_positions(spec) / water.BOHR
    S = system.build_system(spec, pos)
    assert S["natm"] > COUNT_MAX_ATOMS
    box = DeviceBox(S, 1, "fp64")
    d = torch.from_numpy(np.ascontiguousarray(pos[0])).to("cuda:0")
    torch.cuda.synchronize()
    with pytest.raises(PinyError, match=r"count_list_device: ERR_ARG .*PINYB200_COUNT_MAX_ATOMS"):
        box.count_list_device(d.data_ptr(), None, S["hmat"], S["cutskin2"])
    box.close()


def _split_types(F, per_kind=6):
    """The same box with every atom type split into ``per_kind`` types
    (molecule index mod per_kind): the pair set is unchanged, the number of
    pair types ntyp(ntyp+1)/2 grows past the count's fixed limit."""
    from piny_b200.system import _pair_index

    nt0 = int(F["ntyp"])
    nt = nt0 * per_kind
    old = np.repeat(np.arange(nt0), per_kind)          # old type of each new type
    typ0 = np.asarray(F["atm_typ"])
    mol = np.arange(len(typ0)) // 3
    typ = (typ0 * per_kind + mol % per_kind).astype(np.int32)
    npt = nt * (nt + 1) // 2
    imap, cut, cs = np.zeros(npt, np.int32), np.zeros(npt), np.zeros(npt)
    for a in range(nt):
        for b in range(a, nt):
            p, p0 = _pair_index(a, b, nt), _pair_index(old[a], old[b], nt0)
            imap[p], cut[p], cs[p] = F["inter_map"][p0], F["cutoff"][p0], F["cutskin2"][p0]
    G = dict(F)
    G.update(ntyp=nt, atm_typ=typ, inter_map=imap, cutoff=cut, cutskin2=cs)
    return G


def test_count_rejects_too_many_pair_types():
    import torch

    from piny_b200.lib import COUNT_MAX_PAIR_TYPES, DeviceBox, PinyError

    F = load_fixture("spcfw_64_p1")
    G = _split_types(F)
    assert G["ntyp"] * (G["ntyp"] + 1) // 2 > COUNT_MAX_PAIR_TYPES
    box = DeviceBox(G, 1, "fp64")
    # the split box still builds PINY's list through the allocating entry
    assert box.build_list(F["pos"][0], None, G["hmat"], G["cutskin2"]) == F["npairs"]
    d = torch.from_numpy(np.ascontiguousarray(F["pos"][0])).to("cuda:0")
    torch.cuda.synchronize()
    with pytest.raises(PinyError, match=r"count_list_device: ERR_ARG .*PINYB200_COUNT_MAX_PAIR_TYPES"):
        box.count_list_device(d.data_ptr(), None, G["hmat"], G["cutskin2"])
    box.close()
