"""Host-side set-up of one water box for the device force path.

Builds, from a :class:`piny_b200.water.BoxSpec` and bead positions, every
table PINY's input stage builds for its force routines, as plain numpy arrays
in PINY internal units (Bohr, Hartree), 0-based.  The dict keys are the
field names of ``pinyb200_system`` in include/pinyb200.h.  A PINY host fills
the same structure straight from its CLASS/BONDED/GENERAL_DATA instead; this
module is the standalone path.

Each step cites the PINY set-up routine whose arithmetic it restates.
"""
from __future__ import annotations

import math

import numpy as np

from . import water
from .water import BOHR, BOLTZ, KB_KCAL

# PINY's erfc polynomial in t = 1/(1 + 0.3614 x)
# (src/interface/inter_params/spline_fit.c:314-398)
_EP = 0.3614
_E = (0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
      0.4732592578721755, -0.509078520069735, 0.6772631491947646, -0.369912979092217,
      0.06965131976970335)


def _gerfc(tt, eee):
    e1, e2, e3, e4, e5, e6, e7, e8, e9 = _E
    return ((((((((e9 * tt + e8) * tt + e7) * tt + e6) * tt + e5) * tt + e4) * tt + e3) * tt + e2) * tt
            + e1) * tt * eee


def _dgerfc(tt, eee, palp):
    e1, e2, e3, e4, e5, e6, e7, e8, e9 = _E
    d = [1.0 * e1, 2.0 * e2, 3.0 * e3, 4.0 * e4, 5.0 * e5, 6.0 * e6, 7.0 * e7, 8.0 * e8, 9.0 * e9]
    return ((((((((d[8] * tt + d[7]) * tt + d[6]) * tt + d[5]) * tt + d[4]) * tt + d[3]) * tt + d[2]) * tt
             + d[1]) * tt + d[0]) * tt * tt * eee * palp


def nint(x):
    """NINT of PINY (round half away from zero, defines.h:96-97)."""
    x = np.asarray(x, dtype=np.float64)
    return np.where(x >= 0.0, np.trunc(x + 0.5), np.trunc(x - 0.5))


def gethinv(hmat):
    """Inverse and volume of a column-major cell, gethinv order (mathlib.c:353)."""
    h = np.concatenate([[0.0], np.asarray(hmat, np.float64)])
    vol = (h[1] * (h[5] * h[9] - h[8] * h[6]) + h[4] * (h[8] * h[3] - h[2] * h[9])
           + h[7] * (h[2] * h[6] - h[5] * h[3]))
    hi = np.zeros(10)
    hi[1] = (h[5] * h[9] - h[8] * h[6]) / vol
    hi[5] = (h[1] * h[9] - h[7] * h[3]) / vol
    hi[9] = (h[1] * h[5] - h[4] * h[2]) / vol
    hi[4] = (h[7] * h[6] - h[4] * h[9]) / vol
    hi[2] = (h[3] * h[8] - h[2] * h[9]) / vol
    hi[7] = (h[4] * h[8] - h[7] * h[5]) / vol
    hi[3] = (h[2] * h[6] - h[3] * h[5]) / vol
    hi[8] = (h[7] * h[2] - h[8] * h[1]) / vol
    hi[6] = (h[3] * h[4] - h[6] * h[1]) / vol
    return hi[1:], vol


def spline_table(nsplin, rmin, rmax, kind, sig=0.0, eps=0.0, alp=0.0, rheal=1.0, swit=True):
    """spline_vdv (spline_fit.c:28-113): energy and -(1/r)dV/dr tables on
    r_i = dr (i-3) + rmin, i = 1..nsplin, switched over the last ``rheal``."""
    dr = (rmax - rmin) / float(nsplin - 5)
    dri = 1.0 / dr
    i = np.arange(1, nsplin + 1, dtype=np.float64)
    r = dr * (i - 3.0) + rmin
    if swit:
        rp = (r - rmax + rheal) / rheal
        rp = np.minimum(rp, 1.0)
        rp = np.maximum(rp, 0.0)
        sw = 1.0 + rp * rp * (2.0 * rp - 3.0)
        dsw = -6.0 * (rp / rheal) * (rp - 1.0) / r
    else:
        sw = np.ones_like(r)
        dsw = np.zeros_like(r)
    if kind == "null":
        return np.zeros(nsplin), np.zeros(nsplin), dr, dri
    if kind == "lj":
        sig6 = sig * sig * sig * sig * sig * sig
        r2 = r * r
        sig6r = sig6 / (r2 * r2 * r2)
        vnow = (eps * 4. * sig6r * (sig6r - 1.))
        dvnow = (eps * 24. * sig6r * (sig6r * 2. - 1.) / r2)
    elif kind == "coul":
        talp2 = 2.0 * alp * alp
        palp = _EP * alp
        r2 = r * r
        ralp = r * alp
        eee = np.exp(-ralp * ralp)
        tt = 1.0 / (1.0 + _EP * ralp)
        g = _gerfc(tt, eee)
        dg = _dgerfc(tt, eee, palp) + talp2 * g * r
        vnow = 1.0 * g / r
        dvnow = (g / r2 + dg / r) * 1.0 / r
    else:
        raise ValueError(kind)
    return vnow * sw, dvnow * sw + vnow * dsw, dr, dri


def ewald_ecut(kmax, deth):
    """calc_cutoff (set_cp_ewald.c:125-160)."""
    return math.pi * .5 * math.pi * float(kmax * kmax) * math.pow(deth, -(2. / 3.))


def kmaxv_of(ecut, hi):
    out = []
    for d in range(3):
        tr = math.sqrt(hi[d] * hi[d] + hi[d + 3] * hi[d + 3] + hi[d + 6] * hi[d + 6])
        out.append(int(2.0 * (math.sqrt(ecut * .5) / (math.pi * tr))))
    return out


def kvectors(ecut, kmaxv, hi):
    """Half-space spherical k list of countkvec3d/setkvec3d (set_cp_ewald.c:304-586)."""
    tpi = 2.0 * math.pi
    lim = ecut * 4.

    def ktry(a, b, c):
        xk = (a * hi[0] + b * hi[1] + c * hi[2]) * tpi
        yk = (a * hi[3] + b * hi[4] + c * hi[5]) * tpi
        zk = (a * hi[6] + b * hi[7] + c * hi[8]) * tpi
        return (xk * xk + yk * yk + zk * zk) * .5

    kamax = kmaxv[0]
    i = 1
    while i <= kmaxv[0]:
        if ktry(float(i), 0.0, 0.0) > lim:
            break
        i += 1
    kamax = i - 1
    ka_l, kb_l, kc_l = [], [], []
    for ka in range(0, kamax + 1):
        kbmin = 0 if ka == 0 else -kmaxv[1]
        i = kbmin
        while i <= 0:
            if ktry(float(ka), float(i), 0.0) <= lim:
                break
            i += 1
        kbmin = i
        i = 1
        while i <= kmaxv[1]:
            if ktry(float(ka), float(i), 0.0) > lim:
                break
            i += 1
        kbmax = i - 1
        for kb in range(kbmin, kbmax + 1):
            kcmin = 1 if (ka == 0 and kb == 0) else -kmaxv[2]
            i = kcmin
            while i <= 0:
                if ktry(float(ka), float(kb), float(i)) <= lim:
                    break
                i += 1
            kcmin = i
            i = 1
            while i <= kmaxv[2]:
                if ktry(float(ka), float(kb), float(i)) > lim:
                    break
                i += 1
            kcmax = i - 1
            for kc in range(kcmin, kcmax + 1):
                ka_l.append(ka)
                kb_l.append(kb)
                kc_l.append(kc)
    return (np.array(ka_l, np.int32), np.array(kb_l, np.int32), np.array(kc_l, np.int32))


def _radix_ok(n):
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def pme_grid(ecut_now, deth, hi, kmaxv, kmax_pme):
    """set_pme_grid (set_cp_ewald.c:204-300) with radixme's 2^a3^b5^c sizes."""
    ecut_pme = math.pi * .5 * math.pi * float(kmax_pme * kmax_pme) * math.pow(deth, -(2. / 3.))
    ecut = max(ecut_pme, ecut_now)
    temp = []
    for d in range(3):
        tr = math.sqrt(hi[d] * hi[d] + hi[d + 3] * hi[d + 3] + hi[d + 6] * hi[d + 6])
        temp.append(math.sqrt(ecut * .5) / (math.pi * tr))
    while True:
        ng = []
        for d in range(3):
            k = int(nint(temp[d]))
            n = (k + 1) * 4
            while not _radix_ok(n):
                n += 4
            ng.append(n)
        go = False
        for d in range(3):
            if ng[d] < 2 * (kmaxv[d] + 2):
                temp[d] += 1.0
                go = True
        if not go:
            return ng


def bspline_weight_1d(n_interp, ngrid):
    """get_bspline_wght1d (set_cp_ewald.c:1288-1382): 1/|b(m)|^2."""
    mn = np.zeros(n_interp + 1)
    uk = np.zeros(n_interp + 1)
    mn[1] = 1.0
    uk[1] = 1.0
    for k in range(2, n_interp + 1):
        uk[k] = float(k)
    for n in range(3, n_interp + 1):
        rn1 = 1.0 / float(n - 1)
        for k in range(n, 1, -1):
            mn[k] = (uk[k] * mn[k] + (float(n) - uk[k]) * mn[k - 1]) * rn1
        mn[1] = uk[1] * mn[1] * rn1
    grid = float(ngrid)
    tpi_n = 2.0 * math.pi / grid
    m = np.arange(ngrid)
    br = np.zeros(ngrid)
    bi = np.zeros(ngrid)
    for k in range(1, n_interp):
        arg = tpi_n * ((k - 1) * m).astype(np.float64)
        br = br + np.cos(arg) * mn[k]
        bi = bi + np.sin(arg) * mn[k]
    arg = (2.0 * math.pi * float(n_interp - 1) / grid) * m.astype(np.float64)
    nr, ni = np.cos(arg), np.sin(arg)
    den = br * br + bi * bi
    tr = (nr * br + ni * bi) / den
    ti = (ni * br - nr * bi) / den
    return tr * tr + ti * ti


def gauss_legendre_128():
    x, w = np.polynomial.legendre.leggauss(128)
    return x, w


def ecor_table(nsplin, rmax, alp, ecut):
    """splin_ecor (set_exclude.c:548-779): -erf(alpha r)/r plus the finite-k
    Bessel correction, rmin = 0.1 Bohr; also returns self_erf."""
    rmin = 0.1
    dr = (rmax - rmin) / float(nsplin - 5)
    dri = 1.0 / dr
    alp2 = alp * alp
    talp2 = 2.0 * alp * alp
    palp = _EP * alp
    i = np.arange(1, nsplin + 1, dtype=np.float64)
    r12 = dr * (i - 3.0) + rmin
    r12i = 1.0 / r12
    ralp = r12 * alp
    eee = np.exp(-ralp * ralp)
    tt = 1.0 / (1.0 + _EP * ralp)
    temp = _gerfc(tt, eee)
    gerf = 1.0 - temp
    dgerf = _dgerfc(tt, eee, palp) + talp2 * temp * r12
    cv0 = -gerf * r12i
    dvecor = -(dgerf * r12i - gerf / (r12 * r12))
    cdv0 = -dvecor * r12i
    kcut = math.sqrt(2.0 * ecut)
    arg = kcut / (2.0 * alp)
    self_erf = 1.0 - float(_gerfc(1.0 / (1.0 + _EP * arg), math.exp(-arg * arg)))
    kmax = 15.0 * alp
    if kmax > kcut:
        node, weight = gauss_legendre_128()
        dk = kmax - kcut
        pk = kmax + kcut
        know = 0.5 * (node * dk + pk)
        fknow = (dk / math.pi) * np.exp(-0.25 * know * know / alp2) * weight
        a = know[None, :] * r12[:, None]
        s = np.sin(a)
        j0 = s / a
        j1 = (s / a - np.cos(a)) / a
        cv0 = cv0 + (fknow[None, :] * j0).sum(axis=1)
        cdv0 = cdv0 + (know[None, :] * fknow[None, :] * j1 / r12[:, None]).sum(axis=1)
    return cv0, cdv0, dr, dri, self_erf


def ecor_res_table(nsplin, rmax, alp, ecut, ecut_res):
    """ecor.cdv0_res of splin_ecor (set_exclude.c:670-745) for the
    reciprocal-space RESPA set: the force table of ``ecor_table`` without its
    finite-k correction, plus the correction for the RESPA k cutoff
    sqrt(2 ecut_res) (ecut_res = ecor.ecut_res, 4x the RESPA k-list cutoff)."""
    _, cdv0, dr, _, _ = ecor_table(nsplin, rmax, alp, ecut)
    rmin = 0.1
    i = np.arange(1, nsplin + 1, dtype=np.float64)
    r12 = dr * (i - 3.0) + rmin
    node, weight = gauss_legendre_128()
    alp2 = alp * alp
    kmax = 15.0 * alp

    def dchi(kc):
        if not kmax > kc:
            return np.zeros_like(r12)
        dk, pk = kmax - kc, kmax + kc
        know = 0.5 * (node * dk + pk)
        fknow = (dk / math.pi) * np.exp(-0.25 * know * know / alp2) * weight
        a = know[None, :] * r12[:, None]
        s = np.sin(a)
        j1 = (s / a - np.cos(a)) / a
        return (know[None, :] * fknow[None, :] * j1 / r12[:, None]).sum(axis=1)

    return cdv0 - dchi(math.sqrt(2.0 * ecut)) + dchi(math.sqrt(2.0 * ecut_res))


def pme_res_mesh(hmat, kmax_res, kmax_pme_res, n_interp_res):
    """PINY's separate RESPA PME mesh (ewald_respa_pme_opt on,
    control_set_cp_ewald.c:451-504): the RESPA k sphere of ewald_respa_kmax
    (calc_cutoff, countkvec3d / setkvec3d), the mesh of set_pme_grid for
    ewald_respa_kmax_pme, and set_pme_wght's B-spline weights of order
    ewald_respa_interp_pme on that mesh.  ``hmat`` 9 column-major (Bohr).
    Returns the fields of pinyb200_respa's RESPA mesh."""
    hm = np.asarray(hmat, np.float64)
    hi, vol = gethinv(hm)
    ecut = ewald_ecut(int(kmax_res), vol)
    kmaxv = kmaxv_of(ecut, hi)
    ka, kb, kc = kvectors(ecut, kmaxv, hi)
    ng = pme_grid(ecut, vol, hi, kmaxv, int(kmax_pme_res))
    n = int(n_interp_res)
    wa, wb, wc = (bspline_weight_1d(n, g) for g in ng)
    bw = wa[np.where(ka < 0, ka + ng[0], ka)] * wb[np.where(kb < 0, kb + ng[1], kb)] \
        * wc[np.where(kc < 0, kc + ng[2], kc)]
    return {"ngrid_res": np.array(ng, np.int32), "n_interp_res": n, "kastr_res": ka, "kbstr_res": kb,
            "kcstr_res": kc, "bweight_res": bw}


def bend_harm_coefs(fk, theta0):
    """bend_coef "harm" (intra_coefs.c:240-276) and derivatives (:355-371)."""
    cn1, cn2, cn3, cn4 = 49.0 / 72.0, 3.0 / 4.0, 3.0 / 40.0, 1.0 / 180.0
    cn5, cn6, cn7, cn8 = 3.0 / 2.0, 3.0 / 5.0, 1.0 / 10.0, 4.0 / 15.0
    cn9, cn10, cn11 = 8.0 / 45.0, 3.0 / 10.0, 1.0 / 30.0
    c2, c4, c6 = math.cos(2.0 * theta0), math.cos(4.0 * theta0), math.cos(6.0 * theta0)
    s2, s4, s6 = math.sin(2.0 * theta0), math.sin(4.0 * theta0), math.sin(6.0 * theta0)
    c = np.array([0.5 * fk * (cn1 + cn2 * c2 + cn3 * c4 + cn4 * c6), 0.0,
                  0.5 * fk * (-cn5 * c2 - cn6 * c4 - cn7 * c6), 0.0,
                  0.5 * fk * (cn6 * c4 + cn8 * c6), 0.0, 0.5 * fk * (-cn9 * c6)])
    s = np.array([0.0, 0.0, 0.5 * fk * (-cn5 * s2 + cn10 * s4 - cn11 * s6), 0.0,
                  0.5 * fk * (-cn6 * s4 + cn9 * s6), 0.0, 0.5 * fk * (-cn9 * s6)])
    dc = c * np.arange(7.0)
    dc[1] = c[1]
    ds = s * np.array([0.0, 1.0, 1.0, 2.0, 3.0, 4.0, 5.0])
    return c, s, dc, ds


def _pair_index(ti, tj, ntyp):
    i2, i3 = ti + 1, tj + 1
    jj = min(i2, i3)
    ii = i2 + i3 - jj
    return ((jj - 1) * ((ntyp + 1) * 2 - jj)) // 2 + ii - jj


def build_system(spec: "water.BoxSpec", pos_bohr, rheal_A=1.0, hmat=None):
    """Set-up arrays for ``spec`` given bead positions (P, natm, 3) in Bohr;
    ``hmat`` (9, column-major, Bohr) replaces the cubic cell of edge spec.L.

    The bead positions fix the two configuration-dependent set-up values
    PINY derives at start-up: the bead spread that pads the Verlet cutoff
    (get_pimd_spread, pimd_estimators.c:121-220) and the range of the
    Ewald-correction spline (splin_ecor, set_exclude.c:606-621).
    """
    model = spec.model
    nmol = spec.nmol
    ns = model.nsite
    natm = nmol * ns
    pos = np.asarray(pos_bohr, np.float64)
    P = pos.shape[0]
    S = {}
    S["natm"] = natm
    types = model.type_names
    ntyp = len(types)
    S["ntyp"] = ntyp
    site_typ = [types.index(s) for s in model.sites]
    S["atm_typ"] = np.tile(np.array(site_typ, np.int32), nmol)
    S["charge"] = np.tile(np.array(model.charges, np.float64), nmol)

    L = spec.L
    if hmat is None:
        hmat = np.zeros(9)
        hmat[0] = hmat[4] = hmat[8] = L / BOHR
    else:
        hmat = np.array(hmat, np.float64)
    hi, vol = gethinv(hmat)
    S["hmat"] = hmat
    S["hmati"] = hi

    # --- intermolecular tables (set_inter_splin, control_inter_params.c:643)
    npair = ntyp * (ntyp + 1) // 2
    rmin = spec.min_dist / BOHR
    rmax = spec.cutoff / BOHR
    rheal = rheal_A / BOHR
    eps = (model.lj_eps_kcal / KB_KCAL) / BOLTZ
    sig = model.lj_sigma / BOHR
    kinds = []
    for p in range(npair):
        pass
    pair_kind = [None] * npair
    for a in range(ntyp):
        for b in range(a, ntyp):
            pair_kind[_pair_index(a, b, ntyp)] = "lj" if (types[a] == "O" and types[b] == "O") else "null"
    uniq = []
    inter_map = np.zeros(npair, np.int32)
    for p in range(npair):
        if pair_kind[p] not in uniq:
            uniq.append(pair_kind[p])
        inter_map[p] = uniq.index(pair_kind[p])
    kinds = uniq
    S["nsplin"] = spec.nsplin
    S["ninter_unique"] = len(kinds)
    S["inter_map"] = inter_map
    S["cutoff"] = np.full(npair, rmax)
    alp = (spec.alpha * L) / math.pow(vol, 1.0 / 3.0)   # control_set_cp_ewald.c:160-163
    cv0, cdv0, cv0c, cdv0c, rmins, drs, dris = [], [], [], [], [], [], []
    for k in kinds:
        v, dv, dr, dri = spline_table(spec.nsplin, rmin, rmax, k, sig, eps, rheal=rheal)
        vc, dvc, _, _ = spline_table(spec.nsplin, rmin, rmax, "coul", alp=alp, rheal=rheal)
        cv0.append(v)
        cdv0.append(dv)
        cv0c.append(vc)
        cdv0c.append(dvc)
        rmins.append(rmin)
        drs.append(dr)
        dris.append(dri)
    S["rmin_spl"], S["dr_spl"], S["dri_spl"] = np.array(rmins), np.array(drs), np.array(dris)
    S["cv0"], S["cdv0"] = np.concatenate(cv0), np.concatenate(cdv0)
    S["cv0_c"], S["cdv0_c"] = np.concatenate(cv0c), np.concatenate(cdv0c)
    S["skin"] = spec.skin / BOHR
    S["iswit_vdw"] = 1

    # LJ tail (get_clong.c:27-118, swit branch)
    c6 = np.array([(4.0 * eps) * (sig * sig * sig * sig * sig * sig) if pair_kind[p] == "lj" else 0.0
                   for p in range(npair)])
    num = np.bincount(S["atm_typ"], minlength=ntyp)
    cm = np.zeros(npair)
    for a in range(ntyp):
        for b in range(a, ntyp):
            p = _pair_index(a, b, ntyp)
            cm[p] = num[a] * num[b] if a != b else (num[a] * (num[a] - 1)) // 2
    clong = 0.0
    for p in range(npair):
        rc = S["cutoff"][p]
        if c6[p] > 0 and rc - rheal > 0:
            fact = ((1.0 / (rheal * rheal)) * (1.0 / rc + 1.0 / (rc - rheal))
                    + (2.0 / (rheal * rheal * rheal)) * math.log((rc - rheal) / rc))
            clong -= (4.0 * math.pi * c6[p] * cm[p] * fact)
    S["clong"] = clong

    # --- exclusions: every intramolecular pair (set_exclude.c:30-546 for water)
    excl_off = np.zeros(natm + 1, np.int32)
    ej = []
    for i in range(natm):
        m0 = (i // ns) * ns
        js = list(range(m0, i))
        ej.extend(js)
        excl_off[i + 1] = excl_off[i] + len(js)
    S["excl_off"] = excl_off
    S["excl_j"] = np.array(ej, np.int32)

    # --- Ewald / PME (control_set_cp_ewald.c:157-450)
    S["alp_ewd"] = alp
    ecut = ewald_ecut(spec.kmax_ewald, vol)
    kmaxv = kmaxv_of(ecut, hi)
    ka, kb, kc = kvectors(ecut, kmaxv, hi)
    S["nktot"] = len(ka)
    S["kastr"], S["kbstr"], S["kcstr"] = ka, kb, kc
    ng = pme_grid(ecut, vol, hi, kmaxv, spec.kmax_pme)
    S["ngrid_a"], S["ngrid_b"], S["ngrid_c"] = ng
    S["n_interp"] = spec.order
    wa = bspline_weight_1d(spec.order, ng[0])
    wb = bspline_weight_1d(spec.order, ng[1])
    wc = bspline_weight_1d(spec.order, ng[2])
    S["bweight"] = wa[np.where(ka < 0, ka + ng[0], ka)] * wb[np.where(kb < 0, kb + ng[1], kb)] \
        * wc[np.where(kc < 0, kc + ng[2], kc)]

    # --- Ewald exclusion correction: charged excluded pairs
    q = S["charge"]
    j1, j2 = [], []
    for i in range(natm):
        for e in range(excl_off[i], excl_off[i + 1]):
            j = S["excl_j"][e]
            if q[i] != 0.0 and q[j] != 0.0:
                j1.append(i)
                j2.append(j)
    j1 = np.array(j1, np.int32)
    j2 = np.array(j2, np.int32)
    S["necor"] = len(j1)
    S["ecor_j1"], S["ecor_j2"] = j1, j2
    d = pos[:, j1, :] - pos[:, j2, :]
    r2max = float((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]).max()) if len(j1) else 0.0
    ecor_rmax = max(10.0 / BOHR, r2max + 2.0 / BOHR)
    e_cv0, e_cdv0, e_dr, e_dri, self_erf = ecor_table(spec.nsplin, ecor_rmax, alp, 4.0 * ecut)
    S["ecor_nsplin"] = spec.nsplin
    S["ecor_rmin"] = 0.1
    S["ecor_rmax"] = ecor_rmax
    S["ecor_dr"], S["ecor_dri"] = e_dr, e_dri
    S["ecor_cv0"], S["ecor_cdv0"] = e_cv0, e_cdv0
    S["self_erf"] = self_erf

    # --- bonds (O-H1, O-H2) and bends (H1-O-H2): intra_coefs.c
    base = np.arange(nmol, dtype=np.int32) * ns
    S["nbond"] = 2 * nmol
    S["bond_j1"] = np.stack([base, base], axis=1).reshape(-1)
    S["bond_j2"] = np.stack([base + 1, base + 2], axis=1).reshape(-1)
    S["bond_typ"] = np.zeros(2 * nmol, np.int32)
    S["nbond_typ"] = 1
    b = model.bond
    c = np.zeros(7)
    if b["type"] == "harm":
        fk = (b["k"] / KB_KCAL) * (BOHR * BOHR / BOLTZ)
        c[2] = 0.5 * fk
    else:
        D = b["D"] / KB_KCAL
        a = b["a"]
        c[2] = (D * a ** 2) * (math.pow(BOHR, 2.0) / BOLTZ)
        c[3] = (-D * a ** 3) * (math.pow(BOHR, 3.0) / BOLTZ)
        c[4] = (7.0 * D * a ** 4 / 12.0) * (math.pow(BOHR, 4.0) / BOLTZ)
    dc = c * np.arange(7.0)
    dc[1] = c[1]
    S["bond_eq"] = np.array([b["r0"] / BOHR])
    S["bond_c"] = c
    S["bond_dc"] = dc
    S["nbend"] = nmol
    S["bend_j1"] = base + 1
    S["bend_j2"] = base.copy()
    S["bend_j3"] = base + 2
    S["bend_typ"] = np.zeros(nmol, np.int32)
    S["nbend_typ"] = 1
    fkb = (model.bend_k_kcal / KB_KCAL) / BOLTZ
    th0 = model.bend_theta0 * (math.pi / 180.0)
    bc, bs, bdc, bds = bend_harm_coefs(fkb, th0)
    S["bend_eq"] = np.array([th0])
    S["bend_c"], S["bend_s"], S["bend_dc"], S["bend_ds"] = bc, bs, bdc, bds

    # --- ghosts
    if model.ghost:
        g_site, comps = next(iter(model.ghost.items()))
        nc = len(comps)
        S["nghost"] = nmol
        S["ghost_ncomp"] = nc
        S["ghost_atom"] = base + g_site
        S["ghost_comp"] = (base[:, None] + np.array([cidx for cidx, _ in comps], np.int32)[None, :]).reshape(-1)
        S["ghost_coef"] = np.tile(np.array([cf for _, cf in comps]), nmol)
    else:
        S["nghost"] = 0
        S["ghost_ncomp"] = 0

    # --- Verlet cutoff with the bead spread (nbr_list_control.c:249-281)
    if P > 1:
        dd = pos[1:] - pos[:1]
        spread = math.sqrt(float((dd[..., 0] * dd[..., 0] + dd[..., 1] * dd[..., 1]
                                  + dd[..., 2] * dd[..., 2]).max()))
    else:
        spread = 0.0
    S["spread"] = spread
    cs = S["cutoff"] + S["skin"] + spread
    S["cutskin2"] = cs * cs
    return S
