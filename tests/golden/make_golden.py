"""Generate the golden fixtures in tests/golden/ from PINY itself.

Runs PINY's own CPU force path (oracle/_ref/piny_ref, built by
``make -C oracle ref`` from the PINY sources) on seeded synthetic water boxes
and stores, per configuration, a compressed .npz with

* the inputs exactly as PINY used them (bead positions in Bohr after PINY's
  mode round trip, the mode-1 positions for the PIMD image shift, the cell),
* PINY's setup products (spline tables, k list, B-spline weights, exclusion
  and Ewald-correction lists, bond/bend coefficients, ghost definitions),
* PINY's outputs (per-bead forces before and after the M-site
  redistribution, energy components, pressure tensor, the Verlet pair set).

piny_io.npz holds PINY's restart dump and configuration files (text and
binary) for tip4pf_64_p4 with the state they were written from
(``piny_ref io``).  pimd_md.npz holds PINY's Nose-Hoover chain operator and its spring and
centroid-virial routines (``piny_ref nhc`` / ``piny_ref springs``) on seeded
inputs.  It also stores pimd_transforms.npz: PINY's own ring-polymer transforms
(``piny_ref pimd``: path_integral_init, convert_pimd_mode/pos/force_* of
transform_stg.c and transform_cnt.c) of seeded bead positions and forces,
for staging and normal modes at several bead counts.  respa_*.npz hold
PINY's forces at each RESPA level (``piny_ref respa``) for boxes whose inputs
switch the split on.

Run in a container that has the PINY tree:  python tests/golden/make_golden.py
(``--pimd-only`` regenerates just the transform, MD-bookkeeping, I/O and
RESPA fixtures; ``--headline-only`` just the benchmark configurations
evaluated in full: spcfw_256_p32, tip4pf_4096_p32, tip4pf_1024_p16;
``--respa-grid-only`` just the RESPA fixture with PINY's separate RESPA PME
grid)
The GPU tests only read the .npz files.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from piny_b200 import water  # noqa: E402

PINY_REF = os.path.join(ROOT, "oracle", "_ref", "piny_ref")


def read_dump(path):
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


def run_piny(spec, pos_angstrom, workdir):
    d = os.path.join(workdir, "inp")
    shutil.rmtree(d, ignore_errors=True)
    water.write_piny_input(d, spec, pos_angstrom)
    out = os.path.join(workdir, "dump.bin")
    subprocess.run([PINY_REF, "dump", d, "water.input", out], check=True, capture_output=True)
    return read_dump(out)


def pair_hash(pi, pj):
    """Order-independent digest of an (i > j) pair set."""
    key = np.sort(pi.astype(np.int64) * (1 << 32) + pj.astype(np.int64))
    return hashlib.sha256(key.tobytes()).hexdigest()


def dump_to_fixture(D, keep_pairs):
    """PINY dump (1-based) -> fixture dict (0-based, orc_system field names)."""
    n = int(D["natm_tot"][0])
    P = int(D["pi_beads"][0])
    f = {}
    f["natm"] = n
    f["nbeads"] = P
    f["pos"] = D["pos"].reshape(P, n, 3)
    if P > 1:
        f["xmod"] = np.stack([D["xmod"], D["ymod"], D["zmod"]], axis=1)
    f["hmat"] = D["hmat"]
    f["ntyp"] = int(D["natm_typ"][0])
    f["atm_typ"] = D["iatm_atm_typ"] - 1
    f["charge"] = D["q"]
    f["nsplin"] = int(D["nsplin"][0])
    f["ninter_unique"] = int(D["ninter_unique"][0])
    f["inter_map"] = D["inter_map_index"] - 1
    f["cutoff"] = D["cutoff"]
    f["cutskin2"] = D["cutskin"]
    f["rmin_spl"] = D["rmin_spl"]
    f["dr_spl"] = D["dr_spl"]
    f["dri_spl"] = D["dri_spl"]
    for k in ("cv0", "cdv0", "cv0_c", "cdv0_c"):
        f[k] = D[k]
    f["skin"] = float(D["skin"][0])
    f["spread"] = float(D["spread"][0])
    f["clong"] = float(D["clong"][0])
    f["iswit_vdw"] = int(D["iswit_vdw"][0])
    # exclusions as CSR (PINY: excl_num / excl_j_off / excl_j, 1-based)
    num = D["excl_num"]
    off = D["excl_j_off"]
    ej = D["excl_j"] - 1
    excl_off = np.zeros(n + 1, np.int32)
    excl_off[1:] = np.cumsum(num)
    excl_j = np.concatenate([ej[off[i]:off[i] + num[i]] for i in range(n)]) if num.sum() else np.zeros(0, np.int32)
    f["excl_off"] = excl_off
    f["excl_j"] = excl_j.astype(np.int32)
    f["alp_ewd"] = float(D["alp_ewd"][0])
    f["self_erf"] = float(D["self_erf"][0])
    f["nktot"] = int(D["nktot"][0])
    f["kastr"], f["kbstr"], f["kcstr"] = D["kastr"], D["kbstr"], D["kcstr"]
    f["bweight"] = D["bweight_tot"]
    f["ngrid_a"], f["ngrid_b"], f["ngrid_c"] = int(D["ngrid_a"][0]), int(D["ngrid_b"][0]), int(D["ngrid_c"][0])
    f["n_interp"] = int(D["n_interp"][0])
    f["necor"] = int(D["ecor_num"][0])
    f["ecor_j1"] = D["ecor_j1"] - 1
    f["ecor_j2"] = D["ecor_j2"] - 1
    f["ecor_nsplin"] = int(D["ecor_nsplin"][0])
    f["ecor_rmin"] = float(D["ecor_rmin_spl"][0])
    f["ecor_rmax"] = float(D["ecor_rmax_spl"][0])
    f["ecor_dr"] = float(D["ecor_dr_spl"][0])
    f["ecor_dri"] = float(D["ecor_dri_spl"][0])
    f["ecor_ecut"] = float(D["ecor_ecut"][0])
    f["ecor_cv0"] = D["ecor_cv0"]
    f["ecor_cdv0"] = D["ecor_cdv0"]
    f["nbond"] = int(D["bond_npow"][0])
    f["bond_j1"] = D["bond_j1"] - 1
    f["bond_j2"] = D["bond_j2"] - 1
    f["bond_typ"] = D["bond_jtyp"] - 1
    f["nbond_typ"] = int(D["bond_ntyp_pow"][0])
    f["bond_eq"] = D["bond_eq"]
    f["bond_c"] = np.stack([D["bond_c%d" % i] for i in range(7)], axis=1).reshape(-1)
    f["bond_dc"] = np.stack([D["bond_dc%d" % i] for i in range(7)], axis=1).reshape(-1)
    f["nbend"] = int(D["bend_npow"][0])
    f["bend_j1"] = D["bend_j1"] - 1
    f["bend_j2"] = D["bend_j2"] - 1
    f["bend_j3"] = D["bend_j3"] - 1
    f["bend_typ"] = D["bend_jtyp"] - 1
    f["nbend_typ"] = int(D["bend_ntyp_pow"][0])
    f["bend_eq"] = D["bend_eq"]
    f["bend_c"] = np.stack([D["bend_c%d" % i] for i in range(7)], axis=1).reshape(-1)
    f["bend_s"] = np.stack([D["bend_s%d" % i] for i in range(7)], axis=1).reshape(-1)
    # derivative coefficients as bend_coef forms them (intra_coefs.c:355-371)
    c = f["bend_c"].reshape(-1, 7)
    sn = f["bend_s"].reshape(-1, 7)
    dc = c * np.arange(7.0)
    dc[:, 1] = c[:, 1]
    ds = sn * np.array([0.0, 1.0, 1.0, 2.0, 3.0, 4.0, 5.0])
    f["bend_dc"] = dc.reshape(-1)
    f["bend_ds"] = ds.reshape(-1)
    ng = int(D["nghost"][0])
    f["nghost"] = ng
    if ng:
        nc = int(D["ghost_ncomp_max"][0])
        f["ghost_ncomp"] = nc
        f["ghost_atom"] = D["ighost_map"] - 1
        comp = np.full((ng, nc), -1, np.int32)
        coef = np.zeros((ng, nc))
        for c in range(nc):
            comp[:, c] = D["ghost_iatm_%d" % (c + 1)] - 1
            coef[:, c] = D["ghost_coef_%d" % (c + 1)]
        f["ghost_comp"] = comp.reshape(-1)
        f["ghost_coef"] = coef.reshape(-1)
    else:
        f["ghost_ncomp"] = 0
    pairs = D["verlist_pairs"].reshape(-1, 2) - 1
    f["npairs"] = pairs.shape[0]
    f["pairs_sha256"] = pair_hash(pairs[:, 0], pairs[:, 1])
    if keep_pairs:
        f["pairs"] = pairs.astype(np.int32)
    # outputs
    f["ref_force_raw"] = D["force_raw"].reshape(P, n, 3)
    f["ref_force"] = D["force"].reshape(P, n, 3)
    for k in ("vintert", "vintrat", "vvdw", "vcoul", "vrecip", "vlong", "vbondt", "vbendt"):
        f["ref_" + k] = float(D[k][0])
    f["ref_pvten_tot"] = D["pvten_tot"]
    return f


# (name, spec, keep the full pair list in the fixture)
def golden_specs():
    S = water
    return [
        ("spcfw_64_p1", S.BoxSpec(S.SPC_FW, 64, 12.416, 1, 300.0, 101, cutoff=6.0, grid=16, order=6, kmax=6), True),
        ("spcfw_64_p4", S.BoxSpec(S.SPC_FW, 64, 12.416, 4, 300.0, 102, cutoff=6.0, grid=16, order=6, kmax=6), True),
        ("tip4pf_64_p4", S.BoxSpec(S.TIP4P_F, 64, 12.416, 4, 298.0, 103, cutoff=6.0, grid=16, order=8, kmax=6),
         True),
        ("spcfw_256_p1", S.named_spec("spcfw_256_p1"), False),
        ("tip4pf_128_p2", S.BoxSpec(S.TIP4P_F, 128, 15.66, 2, 298.0, 104, cutoff=7.5, grid=24, order=8, kmax=9),
         False),
    ]


PIMD_CASES = [(1, 2), (1, 4), (1, 6), (1, 8), (1, 32), (1, 64), (2, 2), (2, 4), (2, 8), (2, 16), (2, 32), (2, 64)]
PIMD_NATM = 6


def pimd_fixture(tmp):
    """PINY's transforms of seeded ring polymers: per (kind, P) the inputs
    x, f ([P][natm][3]) and PINY's modes, positions back from the modes,
    mode forces, path eigenvalues and bead masses."""
    rng = np.random.default_rng(7)
    mass = np.array([29156.9, 1837.4, 1837.4, 29156.9, 1837.4, 1837.4])[:PIMD_NATM]
    out = {"natm": PIMD_NATM, "mass": mass}
    for kind, P in PIMD_CASES:
        centre = rng.uniform(0.0, 20.0, size=(1, PIMD_NATM, 3))
        x = centre + rng.normal(0.0, 0.3, size=(P, PIMD_NATM, 3))
        f = rng.normal(0.0, 0.05, size=(P, PIMD_NATM, 3))
        inp = os.path.join(tmp, "pimd_in.bin")
        with open(inp, "wb") as fh:
            fh.write(struct.pack("<ii", P, PIMD_NATM))
            fh.write(mass.astype("<f8").tobytes())
            fh.write(x.astype("<f8").tobytes())
            fh.write(f.astype("<f8").tobytes())
        res = os.path.join(tmp, "pimd_out.bin")
        subprocess.run([PINY_REF, "pimd", str(kind), inp, res], check=True, capture_output=True)
        D = read_dump(res)
        tag = "k%d_p%d_" % (kind, P)
        out[tag + "x"] = x
        out[tag + "f"] = f
        for k in ("modes", "back", "fmodes"):
            out[tag + k] = D[k].reshape(P, PIMD_NATM, 3)
        out[tag + "path_eig"] = D["path_eig"]
        out[tag + "bead_mass"] = D["bead_mass"].reshape(P, PIMD_NATM)
        out[tag + "prekf"] = D["prekf"]
    path = os.path.join(HERE, "pimd_transforms.npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in out.items()})
    print("pimd_transforms", os.path.getsize(path), "bytes")


NHC_CASES = [  # (num chains, len, nres, nyosh, shared): shared maps several coordinates to one chain
    (15, 4, 1, 3, False), (2, 2, 2, 5, True), (15, 1, 1, 1, False)]


def pimd_md_fixture(tmp):
    """PINY's chain operator (apply_NHC_par, weights from set_yosh) and its
    spring / centroid-virial routines (mode_energy_control,
    pimd_pvten_forc_corr) on seeded inputs."""
    rng = np.random.default_rng(11)
    n = PIMD_NATM
    out = {"natm": n}
    for c, (num, ln, nres, nyosh, shared) in enumerate(NHC_CASES):
        if shared:  # atoms 0-2 on chain 0, 3-4 on chain 1, atom 5 (a ghost) on the null chain
            per_atom = np.array([1, 1, 1, 2, 2, num + 1])
            inhc = np.tile(per_atom, 3).astype(np.int32)
        else:  # one chain per coordinate of atoms 0-4, atom 5 null
            inhc = np.full(3 * n, num + 1, np.int32)
            for d in range(3):
                inhc[d * n:d * n + 5] = 1 + 3 * np.arange(5) + d
        dti = 41.3 / nres
        m = rng.uniform(1800.0, 30000.0, n)
        v = rng.normal(0.0, 4e-4, (n, 3))
        mass_nhc = rng.uniform(5e3, 5e4, (ln, num))
        gkt = rng.uniform(5e-4, 3e-3, (ln, num))
        x_nhc = rng.normal(0.0, 0.1, (ln, num))
        v_nhc = rng.normal(0.0, 2e-4, (ln, num))
        inp = os.path.join(tmp, "nhc_in.bin")
        with open(inp, "wb") as fh:
            fh.write(struct.pack("<5i", n, num, ln, nres, nyosh))
            fh.write(inhc.astype("<i4").tobytes())
            fh.write(struct.pack("<d", dti))
            for a in (m, v, mass_nhc, gkt, x_nhc, v_nhc):
                fh.write(np.ascontiguousarray(a, "<f8").tobytes())
        res = os.path.join(tmp, "nhc_out.bin")
        subprocess.run([PINY_REF, "nhc", inp, res], check=True, capture_output=True)
        D = read_dump(res)
        t = "nhc%d_" % c
        out.update({t + "num": num, t + "len": ln, t + "nres": nres, t + "nyosh": nyosh, t + "dti": dti,
                    t + "inhc": (inhc - 1).reshape(3, n), t + "mass": m, t + "v": v, t + "mass_nhc": mass_nhc,
                    t + "gkt": gkt, t + "x_nhc": x_nhc, t + "v_nhc": v_nhc, t + "wdti": D["wdti"],
                    t + "ref_v": D["v"].reshape(n, 3), t + "ref_x_nhc": D["x_nhc"].reshape(ln, num),
                    t + "ref_v_nhc": D["v_nhc"].reshape(ln, num)})
    for P in (4, 8):
        T, wght = 300.0, 1.0
        prekf = rng.uniform(1e3, 1e4, n)
        prekf[5] = 0.0
        veig = np.concatenate([[0.0], rng.uniform(1.0, 30.0, P - 1)])
        u = rng.normal(0.0, 0.3, (P, n, 3))
        xmod = rng.uniform(0.0, 20.0, (n, 3))
        x = xmod[None] + rng.normal(0.0, 0.3, (P, n, 3))
        f = rng.normal(0.0, 0.02, (P, n, 3))
        pv, pvt = rng.normal(0.0, 1e-3, 9), rng.normal(0.0, 1e-3, 9)
        inp = os.path.join(tmp, "spr_in.bin")
        with open(inp, "wb") as fh:
            fh.write(struct.pack("<3i", P, n, n))
            fh.write(struct.pack("<2d", T, wght))
            for a in (prekf, veig, u, x, f, xmod, pv, pvt):
                fh.write(np.ascontiguousarray(a, "<f8").tobytes())
        res = os.path.join(tmp, "spr_out.bin")
        subprocess.run([PINY_REF, "springs", inp, res], check=True, capture_output=True)
        D = read_dump(res)
        t = "spr_p%d_" % P
        out.update({t + "T": T, t + "wght": wght, t + "prekf": prekf, t + "veig": veig, t + "u": u, t + "x": x,
                    t + "f": f, t + "xmod": xmod, t + "pvten": pv, t + "pvten_tot": pvt,
                    t + "ref_fm": D["fm"].reshape(P, n, 3), t + "ref_kin_harm": D["kin_harm"][0],
                    t + "ref_pvten_mode_tot": D["pvten_mode_tot"], t + "ref_pvten": D["pvten"],
                    t + "ref_pvten_tot": D["pvten_tot"], t + "ref_akvirx": D["akvirx"][0]})
    path = os.path.join(HERE, "pimd_md.npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in out.items()})
    print("pimd_md", os.path.getsize(path), "bytes")


IO_FILES = ("dump", "conf_pos", "conf_vel", "conf_cent", "conf_force", "conf_par")


def io_fixture(tmp):
    """PINY's restart dump and configuration files (``piny_ref io``: after one
    evaluation of tip4pf_64_p4, write_dump_file_pimd and
    write_config_files_pimd, text and binary) with the state they hold."""
    spec = [s for n, s, k in golden_specs() if n == "tip4pf_64_p4"][0]
    pos = water.build_positions(spec)
    out = {}
    for binary in (0, 1):
        d = os.path.join(tmp, "io_inp%d" % binary)
        shutil.rmtree(d, ignore_errors=True)
        water.write_piny_input(d, spec, pos)
        od = os.path.join(tmp, "io_out%d" % binary)
        shutil.rmtree(od, ignore_errors=True)
        os.makedirs(od)
        subprocess.run([PINY_REF, "io", d, "water.input", od, str(binary)], check=True, capture_output=True)
        if binary == 0:
            D = read_dump(os.path.join(od, "state.bin"))
            for k, v in D.items():
                out["state_" + k] = np.asarray(v)
        for f in IO_FILES:
            if binary == 1 and f == "dump":
                continue
            with open(os.path.join(od, f), "rb") as fh:
                out["file%d_%s" % (binary, f)] = np.frombuffer(fh.read(), np.uint8)
    path = os.path.join(HERE, "piny_io.npz")
    np.savez_compressed(path, **out)
    print("piny_io", os.path.getsize(path), "bytes")


RESPA_CASES = [
    # (name, spec, RESPA keys)
    ("respa_tip4pf_64_p4",
     water.BoxSpec(water.TIP4P_F, 64, 12.416, 4, 298.0, 105, cutoff=6.0, grid=16, order=8, kmax=6),
     {"lrf": 2, "intra": 2, "pimd": 2, "rheal": 0.8, "eq_res": 0.02}),
    ("respa_spcfw_64_p1",
     water.BoxSpec(water.SPC_FW, 64, 12.416, 1, 300.0, 106, cutoff=6.0, grid=16, order=6, kmax=6),
     {"lrf": 3, "intra": 2, "pimd": 1, "rheal": 1.0, "eq_res": -0.01}),
    # the reciprocal-space RESPA set on the one PME grid (PINY demands
    # ewald_respa_kmax = ewald_kmax when ewald_respa_pme_opt is off)
    ("respa_kspace_tip4pf_64_p4",
     water.BoxSpec(water.TIP4P_F, 64, 12.416, 4, 298.0, 107, cutoff=6.0, grid=16, order=8, kmax=6),
     {"lrf": 2, "intra": 2, "pimd": 1, "rheal": 0.8, "eq_res": 0.02, "kmax_res": 6}),
]

# PINY's separate RESPA PME grid (ewald_respa_pme_opt on, kmax_res < kmax,
# kmax_pme_res 4, order 4): the forces of every level and the grid's set-up
# products (mesh, k sphere, B-spline weights, exclusion-correction table)
RESPA_GRID_CASE = ("respa_pmegrid_tip4pf_64_p4",
                   water.BoxSpec(water.TIP4P_F, 64, 12.416, 4, 298.0, 108, cutoff=6.0, grid=16, order=8, kmax=6),
                   {"lrf": 2, "intra": 1, "pimd": 1, "rheal": 0.8, "eq_res": 0.0, "kmax_res": 3, "pme_res": (4, 4)})


def respa_fixture(tmp, cases=None):
    """PINY's forces at each RESPA level (``piny_ref respa``): the flags
    int_NVT_pimd sets at the outer step, an inner inter step, an intra step
    and the innermost step, on seeded boxes with RESPA inputs."""
    for name, spec, rk in (cases if cases is not None else RESPA_CASES + [RESPA_GRID_CASE]):
        pos = water.build_positions(spec)
        d = os.path.join(tmp, "respa_inp")
        shutil.rmtree(d, ignore_errors=True)
        water.write_piny_input(d, spec, pos, respa=rk)
        out = os.path.join(tmp, "respa.bin")
        subprocess.run([PINY_REF, "respa", d, "water.input", out], check=True, capture_output=True)
        D = read_dump(out)
        fx = dump_to_fixture(D, False)
        n, P = fx["natm"], fx["nbeads"]
        for k in ("nres_ter", "nres_tor", "nres_tra", "nres_pimd", "int_res_ter"):
            fx[k] = int(D[k][0])
        for k in ("wght_ter", "wght_ter_res", "wght_tra_res"):
            fx[k] = float(D[k][0])
        fx["cutoff_res"] = D["cutoff_res"]
        fx["rheal_res"] = float(D["rheal_res"][0])
        fx["bond_eq_res"] = D["bond_eq_res"]
        fx["nktot_res"] = int(D["nktot_res"][0])
        fx["pme_res_on"] = int(D["pme_res_on"][0])
        if "ecor_cdv0_res" in D:
            fx["ecor_cdv0_res"] = D["ecor_cdv0_res"]
            fx["ecor_ecut_res"] = float(D["ecor_ecut_res"][0])
        if "ngrid_res" in D:
            fx["kmax_res"] = int(rk["kmax_res"])
            fx["ngrid_res"] = D["ngrid_res"]
            fx["n_interp_res"] = int(D["n_interp_res"][0])
            fx["kmax_pme_res"] = int(D["kmax_pme_res"][0])
            for k in ("kastr_res", "kbstr_res", "kcstr_res", "bweight_tot_res"):
                fx[k] = D[k]
        for lv in range(4):
            fx["L%d_flags" % lv] = D["L%d_flags" % lv]
            fx["ref_L%d_force_raw" % lv] = D["L%d_force_raw" % lv].reshape(P, n, 3)
        if P > 1:
            fx["ref_L0_forcet_raw"] = D["L0_forcet_raw"].reshape(P, n, 3)
        fx["spec_nmol"] = spec.nmol
        fx["spec_L"] = spec.L
        fx["spec_model"] = "tip4pf" if spec.model is water.TIP4P_F else "spcfw"
        fx["spec_cutoff"] = spec.cutoff
        fx["spec_kmax"] = spec.kmax_ewald
        fx["spec_kmax_pme"] = spec.kmax_pme
        fx["spec_order"] = spec.order
        fx["spec_nsplin"] = spec.nsplin
        fx["spec_temperature"] = spec.temperature
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in fx.items()})
        print(name, os.path.getsize(path), "bytes")


# Benchmark configurations evaluated by PINY in full (all beads): the 256
# q-SPC/Fw x 32-bead box, the 4096 q-TIP4P/F x 32-bead box (64^3 mesh, order
# 8) and the 1024 q-TIP4P/F x 16-bead box (32^3 mesh, order 8).
HEADLINE_NAMES = ("spcfw_256_p32", "tip4pf_4096_p32", "tip4pf_1024_p16")


def ulp_offsets(actual, generated):
    """actual - generated in units in the last place (int8), for positions
    PINY used that differ from the seeded generator's by its Angstrom->Bohr
    read and its bead -> mode -> bead round trip."""
    d = actual.view(np.int64) - generated.view(np.int64)
    if np.abs(d).max() > 127:
        raise ValueError("positions differ by more than 127 ulps")
    return d.astype(np.int8)


def headline_fixture(name, tmp):
    """PINY's evaluation of a benchmark configuration, stored compactly: the
    bead positions and mode-1 positions PINY used as ulp offsets from
    water.build_positions (Bohr) and from its bead mean, PINY's raw forces
    (M sites still loaded) of the first and the last bead, every energy
    component (bead averages over all P beads), pvten_tot, the pair count and
    sorted-pair SHA-256 of PINY's Verlet list, PINY's cutskin^2, and digests
    of its set-up (k list SHA-256, every 16th B-spline weight, the spline
    tables)."""
    spec = water.named_spec(name)
    pos_A = water.build_positions(spec)
    D = run_piny(spec, pos_A, tmp)
    n, P = int(D["natm_tot"][0]), int(D["pi_beads"][0])
    gen = pos_A / water.BOHR
    f = {"spec_name": name, "natm": n, "nbeads": P}
    f["pos_ulp"] = ulp_offsets(D["pos"].reshape(P, n, 3), gen)
    if P > 1:
        xm = np.stack([D["xmod"], D["ymod"], D["zmod"]], axis=1)
        f["xmod_ulp"] = ulp_offsets(xm, gen.mean(axis=0))
    f["hmat"] = D["hmat"]
    f["cutskin2"] = D["cutskin"]
    f["spread"] = float(D["spread"][0])
    beads = np.array([0, P - 1]) if P > 1 else np.array([0])
    f["ref_beads"] = beads
    f["ref_force_raw"] = D["force_raw"].reshape(P, n, 3)[beads]
    for k in ("vintert", "vintrat", "vvdw", "vcoul", "vrecip", "vlong", "vbondt", "vbendt"):
        f["ref_" + k] = float(D[k][0])
    f["ref_pvten_tot"] = D["pvten_tot"]
    pairs = D["verlist_pairs"].reshape(-1, 2) - 1
    f["npairs"] = pairs.shape[0]
    f["pairs_sha256"] = pair_hash(pairs[:, 0], pairs[:, 1])
    kv = np.stack([D["kastr"], D["kbstr"], D["kcstr"]], axis=1).astype(np.int32)
    f["nktot"] = int(D["nktot"][0])
    f["kvec_sha256"] = hashlib.sha256(kv.tobytes()).hexdigest()
    f["bweight_every16"] = D["bweight_tot"][::16]
    f["ngrid"] = np.array([int(D["ngrid_a"][0]), int(D["ngrid_b"][0]), int(D["ngrid_c"][0])])
    for k in ("cv0", "cdv0", "cv0_c", "cdv0_c"):
        f[k] = D[k]
    f["inter_map"] = D["inter_map_index"] - 1
    f["alp_ewd"] = float(D["alp_ewd"][0])
    f["clong"] = float(D["clong"][0])
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in f.items()})
    print(name, os.path.getsize(path), "bytes", f["npairs"], "pairs")


def main():
    if "--respa-grid-only" in sys.argv[1:]:
        tmp = tempfile.mkdtemp(prefix="piny_golden_")
        respa_fixture(tmp, [RESPA_GRID_CASE])
        shutil.rmtree(tmp, ignore_errors=True)
        return
    if "--headline-only" in sys.argv[1:]:
        tmp = tempfile.mkdtemp(prefix="piny_golden_")
        for name in HEADLINE_NAMES:
            headline_fixture(name, tmp)
        shutil.rmtree(tmp, ignore_errors=True)
        return
    if not os.path.exists(PINY_REF):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    tmp = tempfile.mkdtemp(prefix="piny_golden_")
    pimd_fixture(tmp)
    pimd_md_fixture(tmp)
    io_fixture(tmp)
    respa_fixture(tmp)
    if "--pimd-only" in sys.argv[1:]:
        shutil.rmtree(tmp, ignore_errors=True)
        return
    for name, spec, keep in golden_specs():
        pos = water.build_positions(spec)
        D = run_piny(spec, pos, tmp)
        fx = dump_to_fixture(D, keep)
        fx["spec_nmol"] = spec.nmol
        fx["spec_L"] = spec.L
        fx["spec_model"] = "tip4pf" if spec.model is water.TIP4P_F else "spcfw"
        fx["spec_cutoff"] = spec.cutoff
        fx["spec_kmax"] = spec.kmax_ewald
        fx["spec_kmax_pme"] = spec.kmax_pme
        fx["spec_order"] = spec.order
        fx["spec_nsplin"] = spec.nsplin
        fx["spec_temperature"] = spec.temperature
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, **{k: np.asarray(v) for k, v in fx.items()})
        print(name, os.path.getsize(out), "bytes", fx["npairs"], "pairs")
    for name in HEADLINE_NAMES:
        headline_fixture(name, tmp)
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
