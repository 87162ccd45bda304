"""Shared test helpers: golden fixtures and box specs."""
import hashlib
import os

import numpy as np

from piny_b200 import water

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_NAMES = ["spcfw_64_p1", "spcfw_64_p4", "tip4pf_64_p4", "spcfw_256_p1", "tip4pf_128_p2"]


def load_fixture(name):
    F = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    return {k: (v.item() if v.ndim == 0 else v) for k, v in F.items()}


def spec_from_fixture(F):
    model = water.TIP4P_F if str(F["spec_model"]) == "tip4pf" else water.SPC_FW
    return water.BoxSpec(model, int(F["spec_nmol"]), float(F["spec_L"]), int(F["nbeads"]),
                         float(F["spec_temperature"]), 0, cutoff=float(F["spec_cutoff"]),
                         grid=int(F["ngrid_a"]), order=int(F["spec_order"]), kmax=int(F["spec_kmax"]),
                         nsplin=int(F["spec_nsplin"]), kmax_pme_in=int(F["spec_kmax_pme"]))


def pair_hash(pi, pj):
    key = np.sort(np.asarray(pi, np.int64) * (1 << 32) + np.asarray(pj, np.int64))
    return hashlib.sha256(key.tobytes()).hexdigest()


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


RESPA_NAMES = ["respa_tip4pf_64_p4", "respa_spcfw_64_p1", "respa_kspace_tip4pf_64_p4", "respa_pmegrid_tip4pf_64_p4"]


def respa_from_fixture(F):
    """pinyb200_set_respa's inputs for a RESPA fixture, formed from its step
    counts the way PINY forms them."""
    from piny_b200 import system
    from piny_b200.respa import respa_setup
    mesh = None
    if int(F.get("pme_res_on", 0)):
        # PINY's separate RESPA PME mesh, set up here as PINY does
        mesh = system.pme_res_mesh(F["hmat"], int(F["kmax_res"]), int(F["kmax_pme_res"]), int(F["n_interp_res"]))
    return respa_setup(int(F["nres_ter"]), int(F["nres_tor"]), int(F["nres_tra"]), int(F["nres_pimd"]),
                       int(F["nbeads"]) > 1, bool(F["int_res_ter"]), F["cutoff_res"], float(F["rheal_res"]),
                       F["bond_eq_res"], nktot_res=int(F["nktot_res"]), ecor_cdv0_res=F.get("ecor_cdv0_res"),
                       mesh_res=mesh)


def fixture_level(F, lv):
    from piny_b200.respa import level_bits
    return level_bits(*[int(v) for v in F["L%d_flags" % lv]])


HEADLINE_NAMES = ["spcfw_256_p32", "tip4pf_4096_p32", "tip4pf_1024_p16"]


def headline_inputs(name):
    """A benchmark configuration exactly as PINY evaluated it: the fixture,
    the spec, the bead positions [P][natm][3] and mode-1 positions (Bohr)
    PINY used -- the seeded generator's positions moved by the stored ulp
    offsets -- and the host set-up built from them."""
    from piny_b200 import system

    F = load_fixture(name)
    spec = water.named_spec(name)
    gen = water.build_positions(spec) / water.BOHR
    pos = (gen.view(np.int64) + F["pos_ulp"].astype(np.int64)).view(np.float64)
    xmod = None
    if "xmod_ulp" in F:
        xmod = (gen.mean(axis=0).view(np.int64) + F["xmod_ulp"].astype(np.int64)).view(np.float64)
    S = system.build_system(spec, pos)
    return F, spec, pos, xmod, S


def read_piny_dump(path):
    """Records of a piny_ref dump file: per record a 32-byte name, a kind
    byte ('d' double, 'i' int32, 'c' text), padding, an int64 count, data."""
    import struct
    out = {}
    with open(path, "rb") as f:
        while True:
            h = f.read(40)
            if len(h) < 40:
                break
            name = h[:32].split(b"\0")[0].decode()
            kind = chr(h[32])
            n = struct.unpack("<q", f.read(8))[0]
            if kind == "c":
                out[name] = f.read(n).decode()
                continue
            dt = np.float64 if kind == "d" else np.int32
            out[name] = np.frombuffer(f.read(n * np.dtype(dt).itemsize), dtype=dt).copy()
    return out
