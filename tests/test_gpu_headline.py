"""The device path at the benchmark configurations against PINY itself.

PINY evaluated each seeded benchmark box in full (tests/golden/*.npz made by
tests/golden/make_golden.py --headline-only): 256 q-SPC/Fw x 32 beads (32^3
mesh), 4096 q-TIP4P/F x 32 beads (64^3 mesh, order 8: the headline
configuration) and 1024 q-TIP4P/F x 16 beads (32^3 mesh).  The device builds
the list from the bead-1 and mode-1 positions PINY used and evaluates all P
beads; the pair set must be PINY's bit for bit, the raw forces of the stored
beads (first and last) within a relative RMS of 1e-12 (FP64) / 1e-5 (MIXED),
and every energy component (bead averages over all P beads) within 1e-11
relative (FP64) / 1e-6 of the summed magnitudes of the terms (MIXED: vintert
is a small difference of large FP32-evaluated sums).
"""
import numpy as np
import pytest

from helpers import HEADLINE_NAMES, headline_inputs, pair_hash, rel_rms

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}
ETOL = {"fp64": 1e-11, "mixed": 1e-6}


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", HEADLINE_NAMES)
def test_device_matches_piny_at_benchmark_size(name, prec):
    from piny_b200.lib import DeviceBox

    F, spec, pos, xmod, S = headline_inputs(name)
    P = int(F["nbeads"])
    box = DeviceBox(S, P, prec)
    n = box.build_list(pos[0], xmod, F["hmat"], F["cutskin2"])
    assert n == F["npairs"]
    gi, gj = box.get_list()
    assert pair_hash(gi, gj) == F["pairs_sha256"]
    f, e = box.energy_force(pos, xmod, F["hmat"])
    beads = F["ref_beads"]
    err = rel_rms(f[beads], F["ref_force_raw"])
    assert err < TOL[prec], err
    scale = 1.0
    if prec == "mixed":
        scale = abs(e["vvdw"]) + abs(e["vcoul"]) + abs(e["vrecip"]) + abs(e["vself"]) + abs(e["vecor"])
    for k, kr in [("vintert", "vintert"), ("vvdw", "vvdw"), ("vcoul", "vcoul"), ("vlong", "vlong"),
                  ("vintrat", "vintrat"), ("vbond", "vbondt"), ("vbend", "vbendt")]:
        ref = F["ref_" + kr]
        assert abs(e[k] - ref) <= ETOL[prec] * max(scale, abs(ref)), (k, e[k], ref)
    vrec = e["vrecip"] + e["vself"] + e["vbgr"] + e["vecor"]
    assert abs(vrec - F["ref_vrecip"]) <= ETOL[prec] * max(scale, abs(F["ref_vrecip"]))
    pv = F["ref_pvten_tot"]
    assert np.abs(e["pvten"] - pv).max() <= ETOL[prec] * 10 * np.abs(pv).max()
    box.close()
