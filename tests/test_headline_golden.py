"""The benchmark configurations against PINY's own evaluation of them.

tests/golden/{spcfw_256_p32, tip4pf_4096_p32, tip4pf_1024_p16}.npz hold
PINY's full evaluation (all beads) of the seeded boxes the benchmark times
(256 q-SPC/Fw x 32 beads on a 32^3 mesh; 4096 q-TIP4P/F x 32 beads on a 64^3
mesh, order 8; 1024 q-TIP4P/F x 16 beads on a 32^3 mesh).  Here, on the CPU:
the host set-up the device path is given (piny_b200.system) equals PINY's at
these sizes, and the oracle reproduces PINY's pair set bit for bit and its
forces of the stored beads (FP64, relative RMS <= 1e-12).  The device path is
held to the same fixtures in test_gpu_headline.py.
"""
import hashlib

import numpy as np
import pytest

from helpers import HEADLINE_NAMES, headline_inputs, pair_hash, rel_rms


@pytest.mark.parametrize("name", HEADLINE_NAMES)
def test_host_setup_matches_piny_at_benchmark_size(name):
    F, spec, pos, xmod, S = headline_inputs(name)
    assert S["natm"] == F["natm"]
    assert np.allclose(S["hmat"], F["hmat"], rtol=1e-15, atol=0)
    assert np.all(np.abs(S["cutskin2"] - F["cutskin2"]) <= 1e-14 * F["cutskin2"])
    assert abs(S["spread"] - F["spread"]) <= 1e-13 * F["spread"]
    assert [S["ngrid_a"], S["ngrid_b"], S["ngrid_c"]] == list(F["ngrid"])
    assert S["nktot"] == F["nktot"]
    kv = np.stack([S["kastr"], S["kbstr"], S["kcstr"]], axis=1).astype(np.int32)
    assert hashlib.sha256(kv.tobytes()).hexdigest() == F["kvec_sha256"]
    assert np.all(np.abs(S["bweight"][::16] - F["bweight_every16"]) <= 1e-14 * F["bweight_every16"])
    assert np.array_equal(S["inter_map"], F["inter_map"])
    for k in ("cv0", "cdv0", "cv0_c", "cdv0_c"):
        ref = F[k]
        assert np.all(np.abs(S[k] - ref) <= 1e-14 * np.maximum(np.abs(ref), 1e-300)), k
    assert abs(S["alp_ewd"] - F["alp_ewd"]) <= 1e-15 * F["alp_ewd"]
    assert abs(S["clong"] - F["clong"]) <= 1e-13 * abs(F["clong"])


@pytest.mark.parametrize("name", HEADLINE_NAMES)
def test_oracle_matches_piny_at_benchmark_size(name, oracle):
    F, spec, pos, xmod, S = headline_inputs(name)
    pi, pj = oracle.verlist(S, pos[0], xmod, F["hmat"], F["cutskin2"])
    assert len(pi) == F["npairs"]
    assert pair_hash(pi, pj) == F["pairs_sha256"]
    beads = F["ref_beads"]
    # per-bead forces depend only on that bead, the list and the mode-1 images
    f, _ = oracle.energy_force(S, pos[beads], xmod, F["hmat"], pi, pj)
    assert rel_rms(f, F["ref_force_raw"]) < 1e-12
