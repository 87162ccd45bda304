"""PINY's restart dump and configuration files (piny_b200.files) against
the files PINY itself wrote (tests/golden/piny_io.npz: ``piny_ref io`` ran
write_dump_file_pimd and write_config_files_pimd after one evaluation of a
64-molecule q-TIP4P/F box with 4 beads, text and binary): the writers
reproduce PINY's bytes from the state PINY held, the readers give that
state back, and reading then writing is the identity on PINY's files."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "piny_io.npz")


@pytest.fixture(scope="module")
def G():
    return np.load(GOLD)


def _state(G):
    names = [tuple(l.split()) for l in str(G["state_names"]).strip().split("\n")]
    cn, cl, bn, bl = (int(x) for x in G["state_nhc_dims"])
    pos = G["state_pos"]
    P = 4
    n = len(names)
    return {
        "pos": pos.reshape(P, n, 3), "vel": G["state_vel"].reshape(P, n, 3), "fxt": G["state_fxt"].reshape(P, n, 3),
        "hmat": G["state_hmat"], "hmat_ewd": G["state_hmat_ewd"], "vgmat": G["state_vgmat"], "names": names,
        "mol_num": G["state_mol_num"], "itime": 0, "class_v_nhc": G["state_class_v_nhc"].reshape(cl, cn),
        "bead_v_nhc": G["state_bead_v_nhc"].reshape(P - 1, bl, bn), "v_lnv": float(G["state_v_lnv"][0]),
        "x_lnv": float(G["state_x_lnv"][0]), "v_vol_nhc": G["state_v_vol_nhc"], "dt": float(G["state_dt"][0]),
        "nfree": int(G["state_nfree"][0]), "ens": G["state_ens"], "free": G["state_free"],
        "t_ext": float(G["state_t_ext"][0]), "pext": float(G["state_pext"][0]),
        "stens_ext": float(G["state_stens_ext"][0])}


def _bytes(path):
    with open(path, "rb") as f:
        return f.read()


def test_dump_writer_reproduces_piny(G, tmp_path):
    from piny_b200 import files
    s = _state(G)
    p = tmp_path / "dump"
    files.write_dump(str(p), s)
    assert _bytes(p) == G["file0_dump"].tobytes()


def test_dump_reader_and_round_trip(G, tmp_path):
    from piny_b200 import files
    s = _state(G)
    src = tmp_path / "piny_dump"
    src.write_bytes(G["file0_dump"].tobytes())
    r = files.read_dump(str(src))
    assert r["restart_typ"] == "restart_all" and r["pi_beads"] == 4 and r["natm"] == len(s["names"])
    for k in ("pos", "vel"):
        assert np.abs(r[k] - s[k]).max() <= 1e-12 * np.abs(s[k]).max()
    for k in ("hmat", "hmat_ewd", "vgmat"):
        assert np.allclose(r[k], s[k], rtol=1e-12, atol=0)
    assert r["names"] == s["names"] and np.array_equal(r["mol_num"], s["mol_num"])
    assert np.allclose(r["class_v_nhc"], s["class_v_nhc"], rtol=1e-12, atol=1e-300)
    assert np.allclose(r["bead_v_nhc"], s["bead_v_nhc"], rtol=1e-9, atol=1e-300)  # PINY writes %.10g
    assert r["dt"] == float("%.13g" % s["dt"]) and r["nfree"] == s["nfree"]
    assert list(r["ens"]) == list(s["ens"]) and list(r["free"]) == list(s["free"])
    out = tmp_path / "again"
    files.write_dump(str(out), r)
    assert _bytes(out) == G["file0_dump"].tobytes()


@pytest.mark.parametrize("binary", [0, 1])
def test_config_writers_reproduce_piny(G, tmp_path, binary):
    from piny_b200 import files
    s = _state(G)
    n = len(s["names"])
    for name, arr in (("conf_pos", s["pos"]), ("conf_vel", s["vel"]), ("conf_force", s["fxt"])):
        p = tmp_path / name
        files.append_config(str(p), arr, s["hmat"], binary=bool(binary))
        assert _bytes(p) == G["file%d_%s" % (binary, name)].tobytes(), name
    p = tmp_path / "conf_par"
    files.append_config(str(p), s["pos"], s["hmat"], binary=bool(binary), lo=2, hi=min(n, 6))
    assert _bytes(p) == G["file%d_conf_par" % binary].tobytes()
    p = tmp_path / "conf_cent"
    files.append_centroid(str(p), s["pos"], s["vel"], s["hmat"], binary=bool(binary))
    assert _bytes(p) == G["file%d_conf_cent" % binary].tobytes()


@pytest.mark.parametrize("binary", [0, 1])
def test_config_reader(G, tmp_path, binary):
    from piny_b200 import files
    s = _state(G)
    n = len(s["names"])
    p = tmp_path / "conf_pos"
    p.write_bytes(G["file%d_conf_pos" % binary].tobytes())
    files.append_config(str(p), s["vel"], s["hmat"], binary=bool(binary))  # a second frame
    fr = files.read_config(str(p), n, 4, binary=bool(binary))
    assert len(fr) == 2
    tol = 0.0 if binary else 1e-11
    for (a, h), want in zip(fr, (s["pos"], s["vel"])):
        assert np.abs(a - want).max() <= tol * np.abs(want).max()
        assert np.allclose(h, s["hmat"], rtol=1e-12, atol=0)
    c = tmp_path / "conf_cent"
    c.write_bytes(G["file%d_conf_cent" % binary].tobytes())
    (cm, v1), h = files.read_config(str(c), n, 4, binary=bool(binary), centroid=True)[0]
    assert np.abs(v1 - s["vel"][0]).max() <= tol * np.abs(s["vel"][0]).max()


def test_initial_file(tmp_path):
    from piny_b200 import files, water
    spec = water.BoxSpec(water.TIP4P_F, 8, water.density_box_edge(8), 2, 298.0, 3, grid=16, order=6)
    pos = water.build_positions(spec)
    d = tmp_path / "inp"
    water.write_piny_input(str(d), spec, pos)
    x, cell, istart = files.read_initial(str(d / "water.initial"), spec.natm, 2)
    assert istart == 1 and x.shape == (2, spec.natm, 3)
    assert np.abs(x * files.BOHR - pos).max() <= 1e-9 * np.abs(pos).max()
    x1, _, _ = files.read_initial(str(d / "water.initial"), spread=True)
    assert x1.shape == (1, spec.natm, 3)


def test_dump_from_a_run_reads_back(tmp_path):
    """A dump written from a run driven here is a restart_all file PINY's
    reader layout accepts (our reader: every field back)."""
    from piny_b200 import files, pimd
    from piny_b200.lib import NORMAL_MODES
    natm, P = 6, 4
    rng = np.random.default_rng(0)
    mass = np.array([29164.4, 1837.5, 1837.5, 29164.4, 1837.5, 1837.5])
    setup = pimd.nvt_setup(mass, None, P, NORMAL_MODES, 300.0, 20.0, 800.0, len_nhc=2)
    pos, vel = rng.normal(size=(P, natm, 3)), rng.normal(size=(P, natm, 3)) * 1e-3
    h = np.diag([20.0, 21.0, 22.0]).reshape(9)
    names = [("O", "water", "water"), ("H", "water", "water"), ("H", "water", "water")] * 2
    s = files.dump_from_run(setup, pos, vel, h, names, [1, 1, 1, 2, 2, 2], itime=7)
    s["class_v_nhc"] = rng.normal(size=(2, 18))
    s["bead_v_nhc"] = rng.normal(size=(P - 1, 2, 18))
    s["v_vol_nhc"] = np.zeros(2)
    p = tmp_path / "dump"
    files.write_dump(str(p), s)
    r = files.read_dump(str(p))
    assert r["itime"] == 7 and r["pi_beads"] == P and r["t_ext"] == 300.0 and r["nfree"] == 18
    assert np.abs(r["pos"] - pos).max() <= 1e-12 and np.abs(r["vel"] - vel).max() <= 1e-15
    assert r["class_v_nhc"].shape == (2, 18) and r["bead_v_nhc"].shape == (P - 1, 2, 18)
