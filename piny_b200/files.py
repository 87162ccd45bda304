"""PINY's coordinate, restart and configuration files (host side).

Readers and writers for the files a PINY run starts from and leaves
behind, so that a run driven by this package (``lib.DevicePimd`` steps on
device arrays) can start from PINY's files and hand its state back to PINY:

* ``read_initial`` -- an ``initial`` start file (read_coord.c:184-199,
  :288-374): ``natm istart pi_beads``, then positions in Angstrom (one
  bead, or every bead), then the cell rows (read but not used by
  read_coord; returned for convenience).
* ``write_dump`` / ``read_dump`` -- the ``restart_all`` dump of
  write_dump_file_pimd (output_pimd.c:786-925): positions with atom,
  residue and molecule names and molecule numbers, the cell and the Ewald
  cell, 1/3 log V, velocities, class and bead chain velocities, cell and
  volume velocities, and the run's time step and ensemble lines.  The
  writer reproduces PINY's bytes (its %.13g / %.10g formats and order);
  the reader accepts PINY's ``restart_pos`` / ``restart_posvel`` /
  ``restart_all`` files (read_coord.c:202-260, :376-900).
* ``append_config`` / ``read_config`` -- the configuration trajectories
  of write_config_files_pimd (output_pimd.c:1093-1340): bead positions
  (or velocities, or forces) per frame followed by the cell rows, as text
  (%.12g, cell %.13g) or binary doubles; ``append_centroid`` the centroid
  file (bead-averaged positions and bead-1 velocities).

Arrays are bead-major [P][natm][3] in Bohr (PINY's internal units), cells
are 9 numbers in PINY's ``hmat[1..9]`` order (column-major).
"""
from __future__ import annotations

import math
import os

import numpy as np

BOHR = 0.529177  # Angstrom per Bohr (PINY defines.h)


def _g(fmt, *v):
    return fmt % v


def _hrows(h, fmt="%.13g"):
    """Cell rows as PINY writes them: row i = hmat[1+i], hmat[4+i], hmat[7+i]."""
    h = np.asarray(h, np.float64).reshape(9)
    return ["%s %s %s" % (fmt % h[i], fmt % h[3 + i], fmt % h[6 + i]) for i in range(3)]


def getdeth(h):
    """Determinant of PINY's cell in its operation order (mathlib.c:433-444)."""
    h = [float(x) for x in np.asarray(h, np.float64).reshape(9)]
    return (h[0] * (h[4] * h[8] - h[7] * h[5]) + h[3] * (h[7] * h[2] - h[1] * h[8]) +
            h[6] * (h[1] * h[5] - h[4] * h[2]))


def read_initial(path, natm=None, pi_beads=None, spread=False):
    """An ``initial`` start file: (pos [P'][natm][3] Bohr, cell rows in
    Angstrom [3][3], istart).  spread=True reads one bead (PINY's
    initial_spread_opt), else every bead."""
    with open(path) as f:
        head = f.readline().split()
        n, istart, P = int(head[0]), int(head[1]), int(head[2])
        if natm is not None and n != natm:
            raise ValueError("%s: %d atoms, expected %d" % (path, n, natm))
        if pi_beads is not None and P != pi_beads:
            raise ValueError("%s: %d beads, expected %d" % (path, P, pi_beads))
        nb = 1 if spread else P
        pos = np.empty((nb, n, 3))
        for b in range(nb):
            for i in range(n):
                t = f.readline().split()
                pos[b, i] = [float(t[0]) / BOHR, float(t[1]) / BOHR, float(t[2]) / BOHR]
        cell = np.array([[float(x) for x in f.readline().split()[:3]] for _ in range(3)])
    return pos, cell, istart


def write_dump(path, s):
    """PINY's ``restart_all`` dump (write_dump_file_pimd).  ``s`` holds pos,
    vel ([P][natm][3]), hmat, hmat_ewd, vgmat (9 each), names (per atom
    (atm, res, mol)), mol_num, itime, class_v_nhc [len][num], bead_v_nhc
    [P-1][len][num], v_lnv, v_vol_nhc [len], dt, nfree, ens (nve, nvt,
    npt_i, npt_f, nst), free (bond, bend, tors), t_ext, pext, stens_ext; and
    x_lnv when npt_i is on (else 1/3 log det h, with v_lnv the mean of
    vgmat's diagonal, as PINY sets them)."""
    pos = np.asarray(s["pos"], np.float64)
    vel = np.asarray(s["vel"], np.float64)
    P, n = pos.shape[0], pos.shape[1]
    names, mol_num = s["names"], np.asarray(s["mol_num"])
    vg = np.asarray(s["vgmat"], np.float64).reshape(9)
    ens = [int(x) for x in s["ens"]]
    if ens[2] == 0:
        x_lnv = math.log(getdeth(s["hmat"])) / 3.0
        v_lnv = (float(vg[0]) + float(vg[4]) + float(vg[8])) / 3.0
    else:
        x_lnv, v_lnv = float(s["x_lnv"]), float(s["v_lnv"])
    cv = np.asarray(s["class_v_nhc"], np.float64)
    bv = np.asarray(s["bead_v_nhc"], np.float64)
    out = ["natm_tot restart_typ itime pi_beads", "%d restart_all %d %d" % (n, int(s["itime"]), P),
           "atm pos, atm_typ, mol_typ mol_num"]
    for b in range(P):
        for i in range(n):
            a, r, m = names[i]
            out.append("%.13g %.13g %.13g %s %s %s %d" % (pos[b, i, 0], pos[b, i, 1], pos[b, i, 2], a, r, m,
                                                         int(mol_num[i])))
    out.append("h matrix")
    out += _hrows(s["hmat"])
    out.append("h matrix for Ewald setup")
    out += _hrows(s["hmat_ewd"])
    out.append("1/3 log(Vol)")
    out.append("%.13g" % x_lnv)
    out.append("atm vel")
    for b in range(P):
        for i in range(n):
            out.append("%.13g %.13g %.13g" % (vel[b, i, 0], vel[b, i, 1], vel[b, i, 2]))
    out.append("number of atm nhc, length of nhc")
    clen, cnum = (cv.shape if cv.size else (0, 0))
    out.append("%d %d" % (cnum, clen))
    out.append("atm nhc velocities")
    out += ["%.13g" % x for x in cv.reshape(-1)]
    out.append("number of bead nhc, length of nhc")
    blen, bnum = (bv.shape[1], bv.shape[2]) if bv.ndim == 3 else (int(s.get("bead_len", 0)), int(s.get("bead_num", 0)))
    out.append("%d %d" % (bnum, blen))
    out.append("bead nhc velocities")
    out += ["%.10g" % x for x in bv.reshape(-1)]
    out.append("vol velocities")
    out += _hrows(vg)
    out.append("log(vol) velocity")
    out.append("%.13g" % v_lnv)
    out.append("vol nhc velocities")
    out += ["%.13g" % x for x in np.asarray(s["v_vol_nhc"], np.float64).reshape(-1)]
    out.append("dt=%.13g" % float(s["dt"]))
    out.append("nfree=%d" % int(s["nfree"]))
    out.append("nve=%d nvt=%d npt_i=%d npt_f=%d nst=%d" % tuple(ens))
    out.append("nbond_free=%d nbend_free=%d ntors_free=%d" % tuple(int(x) for x in s["free"]))
    out.append("t_ext=%.13g,pext=%.13g,stens_ext=%.13g" % (float(s["t_ext"]), float(s["pext"]),
                                                            float(s["stens_ext"])))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def _rows(lines, k, n):
    return [lines[k + i].split() for i in range(n)], k + n


def read_dump(path, natm=None):
    """A PINY restart file (restart_pos, restart_posvel or restart_all) as
    the dict ``write_dump`` takes; parts the file does not hold are left
    out.  Positions and velocities in Bohr and atomic units, as PINY keeps
    them."""
    with open(path) as f:
        lines = f.read().split("\n")
    h = lines[1].split()
    n, kind, itime, P = int(h[0]), h[1], int(h[2]), int(h[3])
    if natm is not None and n != natm:
        raise ValueError("%s: %d atoms, expected %d" % (path, n, natm))
    s = {"natm": n, "restart_typ": kind, "itime": itime, "pi_beads": P}
    k = 3
    rows, k = _rows(lines, k, P * n)
    s["pos"] = np.array([[float(r[0]), float(r[1]), float(r[2])] for r in rows]).reshape(P, n, 3)
    s["names"] = [(r[3], r[4], r[5]) for r in rows[:n]]
    s["mol_num"] = np.array([int(r[6]) for r in rows[:n]])

    def cell(k):
        r, k = _rows(lines, k + 1, 3)
        m = np.array([[float(x) for x in row[:3]] for row in r])
        return m.T.reshape(9), k  # rows back to PINY's column-major hmat

    s["hmat"], k = cell(k)
    s["hmat_ewd"], k = cell(k)
    s["x_lnv"] = float(lines[k + 1])
    k += 2
    if kind in ("restart_posvel", "restart_all"):
        rows, k = _rows(lines, k + 1, P * n)
        s["vel"] = np.array([[float(x) for x in r[:3]] for r in rows]).reshape(P, n, 3)
    if kind == "restart_all":
        cnum, clen = (int(x) for x in lines[k + 1].split()[:2])
        vals, k = _rows(lines, k + 3, cnum * clen)
        s["class_v_nhc"] = np.array([float(r[0]) for r in vals]).reshape(clen, cnum)
        bnum, blen = (int(x) for x in lines[k + 1].split()[:2])
        vals, k = _rows(lines, k + 3, (P - 1) * bnum * blen)
        s["bead_v_nhc"] = np.array([float(r[0]) for r in vals]).reshape(P - 1, blen, bnum)
        vg, k = cell(k)
        s["vgmat"] = vg
        s["v_lnv"] = float(lines[k + 1])
        k += 2
        vals, k = _rows(lines, k + 1, clen)
        s["v_vol_nhc"] = np.array([float(r[0]) for r in vals])
        s["dt"] = float(lines[k].split("=")[1])
        s["nfree"] = int(lines[k + 1].split("=")[1])
        s["ens"] = [int(t.split("=")[1]) for t in lines[k + 2].split()]
        s["free"] = [int(t.split("=")[1]) for t in lines[k + 3].split()]
        te = dict(t.split("=") for t in lines[k + 4].split(","))
        s["t_ext"], s["pext"], s["stens_ext"] = float(te["t_ext"]), float(te["pext"]), float(te["stens_ext"])
    return s


def append_config(path, arr, hmat, binary=False, lo=None, hi=None):
    """One frame of a configuration file (positions, velocities or forces):
    every bead's rows, then the cell rows.  lo/hi (1-based, inclusive)
    write PINY's partial file (atoms lo..hi)."""
    a = np.asarray(arr, np.float64)
    if lo is not None:
        a = a[:, lo - 1:hi, :]
    h = np.asarray(hmat, np.float64).reshape(9)
    hr = np.array([[h[i], h[3 + i], h[6 + i]] for i in range(3)])
    if binary:
        with open(path, "ab") as f:
            f.write(np.ascontiguousarray(a).astype("<f8").tobytes())
            f.write(hr.astype("<f8").tobytes())
        return
    out = ["%.12g  %.12g  %.12g" % tuple(r) for r in a.reshape(-1, 3)]
    out += _hrows(h)
    with open(path, "a") as f:
        f.write("\n".join(out) + "\n")


def append_centroid(path, pos, vel, hmat, binary=False):
    """One frame of PINY's centroid file: bead-averaged positions (summed
    over beads in bead order, then divided), bead-1 velocities, cell rows."""
    pos = np.asarray(pos, np.float64)
    P = pos.shape[0]
    cm = np.zeros(pos.shape[1:])
    for b in range(P):
        cm = cm + pos[b]
    cm = cm / float(P)
    v1 = np.asarray(vel, np.float64)[0]
    h = np.asarray(hmat, np.float64).reshape(9)
    if binary:
        hr = np.array([[h[i], h[3 + i], h[6 + i]] for i in range(3)])
        with open(path, "ab") as f:
            f.write(cm.astype("<f8").tobytes())
            f.write(v1.astype("<f8").tobytes())
            f.write(hr.astype("<f8").tobytes())
        return
    out = ["%.12g  %.12g  %.12g" % tuple(r) for r in cm]
    out += ["%.12g  %.12g  %.12g" % tuple(r) for r in v1]
    out += _hrows(h)
    with open(path, "a") as f:
        f.write("\n".join(out) + "\n")


def read_config(path, natm, pi_beads, binary=False, centroid=False):
    """Frames of a configuration file: list of (array, hmat).  For the
    centroid file each frame is ((centroid positions, bead-1 velocities),
    hmat)."""
    rows_per = 2 * natm if centroid else pi_beads * natm
    frames = []
    if binary:
        data = np.fromfile(path, dtype="<f8")
        per = 3 * rows_per + 9
        for f0 in range(0, data.size - per + 1, per):
            blk = data[f0:f0 + per]
            hr = blk[3 * rows_per:].reshape(3, 3)
            a = blk[:3 * rows_per].reshape(-1, 3)
            frames.append(((a[:natm], a[natm:]) if centroid else a.reshape(pi_beads, natm, 3), hr.T.reshape(9)))
        return frames
    with open(path) as f:
        lines = [l for l in f.read().split("\n") if l.strip()]
    per = rows_per + 3
    for f0 in range(0, len(lines) - per + 1, per):
        a = np.array([[float(x) for x in l.split()] for l in lines[f0:f0 + rows_per]])
        hr = np.array([[float(x) for x in l.split()] for l in lines[f0 + rows_per:f0 + per]])
        frames.append(((a[:natm], a[natm:]) if centroid else a.reshape(pi_beads, natm, 3), hr.T.reshape(9)))
    return frames


def dump_from_run(setup, pos, vel, hmat, names, mol_num, itime=0, pimd=None, t_ext=None, dt=None):
    """A write_dump state for a run driven here (``pimd.nvt_setup``'s
    ``setup``): chain velocities read from a ``lib.DevicePimd`` (pimd),
    everything volume-related zero (NVT), nfree = 3 per non-ghost atom (PINY's
    count without constraints)."""
    P, n = np.asarray(pos).shape[:2]
    cv = bv = np.zeros((0, 0))
    if pimd is not None:
        cx, cvv = pimd.get_nhc(0)
        bx, bvv = pimd.get_nhc(1)
        cv = cvv if cvv is not None else cv
        bv = bvv if bvv is not None else np.zeros((P - 1, 0, 0))
    clen = cv.shape[0] if cv.size else 0
    return {"pos": pos, "vel": vel, "hmat": hmat, "hmat_ewd": hmat, "vgmat": np.zeros(9), "names": names,
            "mol_num": mol_num, "itime": itime, "class_v_nhc": cv, "bead_v_nhc": bv, "v_vol_nhc": np.zeros(clen),
            "dt": setup["dt"] if dt is None else dt, "nfree": int(setup.get("nfree_atoms", n)) * 3,
            "ens": (0, 1, 0, 0, 0), "free": (0, 0, 0),
            "t_ext": (setup.get("temperature", 0.0) if t_ext is None else t_ext), "pext": 0.0, "stens_ext": 0.0}
