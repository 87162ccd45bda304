"""PINY itself, with its three force sub-steps bound to the library.

oracle/_ref/piny_ref_gpu is PINY's own code (parse, get_ghost_pos,
energy_control_initial, list test, stat_avg bookkeeping, distrib_ghost_force)
with energy_control_inter_real / _inter_recip / _intra replaced by the
binding in oracle/ref/energy_control_gpu.c: gpu_force_init turns PINY's
CLASS / BONDED / GENERAL_DATA into a library context, gpu_energy_control
runs PINY's list test and the device evaluation of all beads.  It is
compared with oracle/_ref/piny_ref (PINY unmodified) on the same input
directory: Verlet pair sets equal, forces (raw, virial, after PINY's ghost
redistribution) within a relative RMS of 1e-12 (FP64) / 1e-5 (MIXED),
energies and pressure tensors within 1e-11 relative (FP64) / 1e-6 of the
summed magnitudes of the terms the total is a difference of (MIXED: FP32
pair sums over millions of pairs carry ~1e-5 absolute rounding), and no
rebuild on a second call with the same positions.
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import pair_hash, read_piny_dump, rel_rms

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF = os.path.join(ROOT, "oracle", "_ref", "piny_ref")
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "piny_ref_gpu")


def _spec(name):
    from piny_b200 import water
    if name == "tip4pf_64_p4":
        return water.BoxSpec(water.TIP4P_F, 64, 12.416, 4, 298.0, 103, cutoff=6.0, grid=16, order=8, kmax=6)
    return water.named_spec(name)


@pytest.fixture(scope="module")
def cpu_dumps(tmp_path_factory):
    if not (os.path.exists(REF) and os.path.exists(REF_GPU)):
        pytest.skip("PINY builds (make -C oracle ref ref-gpu) are not present")
    return {}


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["tip4pf_64_p4", "spcfw_256_p1", "tip4pf_1024_p16", "tip4pf_4096_p32"])
def test_piny_with_gpu_binding_matches_piny(name, prec, cpu_dumps, tmp_path):
    from piny_b200 import water
    spec = _spec(name)
    pos = water.build_positions(spec)
    # one input directory per run: PINY will not overwrite the output files
    # an earlier run left there
    if name not in cpu_dumps:
        dc = tmp_path / "inp_cpu"
        water.write_piny_input(str(dc), spec, pos)
        out = str(tmp_path / "cpu.bin")
        subprocess.run([REF, "dump", str(dc), "water.input", out], check=True, capture_output=True)
        cpu_dumps[name] = read_piny_dump(out)
    C = cpu_dumps[name]
    d = tmp_path / "inp_gpu"
    water.write_piny_input(str(d), spec, pos)
    out = str(tmp_path / "gpu.bin")
    r = subprocess.run([REF_GPU, "gpu_dump", str(d), "water.input", out, "1" if prec == "mixed" else "0"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    G = read_piny_dump(out)
    cp = C["verlist_pairs"].reshape(-1, 2)
    gp = G["gpu_pairs"].reshape(-1, 2)
    assert len(gp) == len(cp)
    assert pair_hash(gp[:, 0], gp[:, 1]) == pair_hash(cp[:, 0], cp[:, 1])
    assert float(G["gpu_rebuilds_second_call"][0]) == 0.0
    tol = {"fp64": 1e-12, "mixed": 1e-5}[prec]
    for k in ("force_raw", "force") + (("forcet_raw",) if "forcet_raw" in C else ()):
        assert rel_rms(G[k], C[k]) < tol, k
    scale = 1.0
    if prec == "mixed":
        # the summed magnitudes of the terms vintert is a difference of, as the
        # other MIXED parity tests take them: vdW, real-space and reciprocal
        # Ewald, the LJ tail and the Ewald self term (ewald3d_self_bgr.c:28-80)
        vself = float(C["alp_ewd"][0] * C["self_erf"][0] * np.sum(C["q"] ** 2) / np.sqrt(np.pi))
        scale = abs(C["vvdw"][0]) + abs(C["vcoul"][0]) + abs(C["vrecip"][0]) + abs(C["vlong"][0]) + vself
    etol = {"fp64": 1e-11, "mixed": 1e-6}[prec]
    for k in ("vintert", "vintrat", "vvdw", "vcoul", "vrecip", "vlong", "vbondt", "vbendt"):
        ref = float(C[k][0])
        assert abs(float(G[k][0]) - ref) <= etol * max(scale, abs(ref)), (k, float(G[k][0]), ref)
    for k in ("pvten_tot", "pvten"):
        assert np.abs(G[k] - C[k]).max() <= etol * 10 * np.abs(C[k]).max(), k
