"""Parameter tangents of the host set-up (piny_b200.params.tangents)
against central differences of piny_b200.system.build_system, and the
parameter vector round trip.  No GPU."""
import dataclasses

import numpy as np

from piny_b200 import params, system, water

KEYS = {"charge": "dcharge", "ghost_coef": "dghost_coef", "cv0": "dcv0", "cdv0": "dcdv0", "bond_c": "dbond_c",
        "bond_eq": "dbond_eq", "bend_c": "dbend_c", "bend_s": "dbend_s", "bend_dc": "dbend_dc",
        "bend_ds": "dbend_ds", "clong": "dclong"}


def test_theta_round_trip():
    th = params.theta_of(water.TIP4P_F)
    assert len(th) == len(params.PARAMS)
    m = params.model_with(water.TIP4P_F, th)
    assert np.allclose(params.theta_of(m), th)
    assert m.charges[3] == -2 * m.charges[1]
    assert abs(sum(c for _, c in m.ghost[3]) - 1.0) < 1e-15


def test_tangents_match_finite_differences_of_the_setup():
    spec = water.BoxSpec(water.TIP4P_F, 64, water.density_box_edge(64), 2, 298.0, 3, grid=16, order=8)
    pos = water.build_positions(spec) / water.BOHR
    th = params.theta_of(spec.model)

    def setup(t):
        return system.build_system(dataclasses.replace(spec, model=params.model_with(spec.model, t)), pos)

    tans = params.tangents(spec, th, setup(th))
    for k in range(len(th)):
        h = 1e-6 * abs(th[k])
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        Sp, Sm = setup(tp), setup(tm)
        for key, tk in KEYS.items():
            fd = (np.asarray(Sp[key], float) - np.asarray(Sm[key], float)) / (2 * h)
            an = np.asarray(tans[k].get(tk, 0.0), float)
            scale = max(np.abs(fd).max(), np.abs(an).max(), 1e-300)
            assert np.abs(fd - an).max() <= 1e-7 * scale, (params.PARAMS[k], key)
