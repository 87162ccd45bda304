"""Parameter gradients (pinyb200_grad) of q-TIP4P/F.

theta = (qH, gamma, sigma, epsilon, D, a, r0, k_bend, theta0).  The FP64
adjoint is checked against central finite differences (h = 1e-5 relative)
of the oracle's energy and of a force-matching loss sum |F - F_target|^2,
F_target from the same configuration with every parameter perturbed by
seeded +-2 %; the MIXED adjoint against the FP64 one.

Tolerances: FP64 adjoint vs finite differences 2e-6 relative per
component for every parameter but gamma, and 2e-5 of the largest component
for all (gamma's differences scatter by ~1 %: see the last test); MIXED vs
FP64 1e-3 of the largest component.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _box():
    from piny_b200 import water
    spec = water.BoxSpec(water.TIP4P_F, 128, water.density_box_edge(128), 2, 298.0, 31, grid=16, order=8)
    return spec, water.build_positions(spec)


def _oracle_eval(oracle, spec, pos_A, theta, pi=None, pj=None):
    from piny_b200 import params, system, water
    sp = dataclasses.replace(spec, model=params.model_with(spec.model, theta))
    pos = pos_A / water.BOHR
    S = system.build_system(sp, pos)
    xmod = pos.mean(axis=0)
    if pi is None:
        pi, pj = oracle.verlist(S, pos[0], xmod, S["hmat"], S["cutskin2"])
    f, e = oracle.energy_force(S, pos, xmod, S["hmat"], pi, pj, distribute_ghosts=True)
    return e["vintert"] + e["vintrat"], f, pi, pj


def _fd(oracle, spec, pos_A, theta, f_target, pi, pj):
    gE, gL = np.zeros(len(theta)), np.zeros(len(theta))
    for k in range(len(theta)):
        h = 1e-5 * abs(theta[k])
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        Ep, Fp, _, _ = _oracle_eval(oracle, spec, pos_A, tp, pi, pj)
        Em, Fm, _, _ = _oracle_eval(oracle, spec, pos_A, tm, pi, pj)
        gE[k] = (Ep - Em) / (2 * h)
        gL[k] = (((Fp - f_target) ** 2).sum() - ((Fm - f_target) ** 2).sum()) / (2 * h)
    return gE, gL


@pytest.fixture(scope="module")
def problem(oracle):
    from piny_b200 import params
    spec, pos_A = _box()
    theta = params.theta_of(spec.model)
    rng = np.random.default_rng(2024)
    theta_t = theta * (1.0 + rng.uniform(-0.02, 0.02, size=theta.shape))
    _, f_target, pi, pj = _oracle_eval(oracle, spec, pos_A, theta_t)
    E, F, pi, pj = _oracle_eval(oracle, spec, pos_A, theta, pi, pj)
    gE, gL = _fd(oracle, spec, pos_A, theta, f_target, pi, pj)
    return spec, pos_A, theta, f_target, E, F, gE, gL


def _adjoint(spec, pos_A, theta, f_target, precision):
    from piny_b200.params import PinyForceField
    field = PinyForceField(spec, pos_A, precision)
    E, F = field.energy_forces(theta)
    fbar = 2.0 * (F - f_target)
    gE = field.adjoint(theta, 1.0, None)
    gL = field.adjoint(theta, 0.0, fbar)
    field.close()
    return E, F, gE, gL


def test_fp64_adjoint_matches_finite_differences(problem):
    spec, pos_A, theta, f_target, E0, F0, gE_fd, gL_fd = problem
    E, F, gE, gL = _adjoint(spec, pos_A, theta, f_target, "fp64")
    assert abs(E - E0) <= 1e-11 * abs(E0)
    assert np.linalg.norm(F - F0) <= 1e-12 * np.linalg.norm(F0)
    from piny_b200.params import PARAMS
    sE, sL = np.abs(gE_fd).max(), np.abs(gL_fd).max()
    for k in range(len(theta)):
        assert abs(gE[k] - gE_fd[k]) <= 2e-5 * sE, ("dE", k, gE[k], gE_fd[k])
        assert abs(gL[k] - gL_fd[k]) <= 2e-5 * sL, ("dL", k, gL[k], gL_fd[k])
        if PARAMS[k] != "gamma":
            assert abs(gE[k] - gE_fd[k]) <= 2e-6 * abs(gE_fd[k]), ("dE", PARAMS[k], gE[k], gE_fd[k])
            assert abs(gL[k] - gL_fd[k]) <= 2e-6 * abs(gL_fd[k]), ("dL", PARAMS[k], gL[k], gL_fd[k])


def test_mixed_adjoint_matches_fp64(problem):
    spec, pos_A, theta, f_target, *_ = problem
    _, _, gE64, gL64 = _adjoint(spec, pos_A, theta, f_target, "fp64")
    _, _, gE32, gL32 = _adjoint(spec, pos_A, theta, f_target, "mixed")
    assert np.abs(gE32 - gE64).max() <= 1e-3 * np.abs(gE64).max()
    assert np.abs(gL32 - gL64).max() <= 1e-3 * np.abs(gL64).max()


def test_autograd_function(problem):
    import torch

    from piny_b200.params import PinyForceField, energy_forces
    spec, pos_A, theta, f_target, E0, F0, gE_fd, gL_fd = problem
    field = PinyForceField(spec, pos_A, "fp64")
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    E, F = energy_forces(th, field)
    loss = E + ((F - torch.from_numpy(f_target)) ** 2).sum()
    loss.backward()
    want = gE_fd + gL_fd
    assert np.abs(th.grad.numpy() - want).max() <= 2e-5 * np.abs(want).max()
    field.close()


def test_grad_call_order_and_limits():
    from piny_b200.lib import DeviceBox, PinyError
    from piny_b200 import system, water
    spec, pos_A = _box()
    pos = pos_A / water.BOHR
    S = system.build_system(spec, pos)
    box = DeviceBox(S, spec.nbeads, "fp64")
    box.build_list(pos[0], pos.mean(axis=0), S["hmat"], S["cutskin2"])
    import torch
    d = torch.from_numpy(pos).to("cuda:0")
    with pytest.raises(PinyError, match="ERR_STATE"):
        box.grad(d.data_ptr(), None, S["hmat"])
    with pytest.raises(PinyError, match="ERR_ARG"):
        box.grad_prepare([{"dclong": 0.0}] * 17)
    box.close()


def test_ghost_parameter_without_tabulated_coulomb(oracle):
    """gamma moves the M sites, so its force-matching gradient goes through
    Hessian-vector products.  PINY's real-space Coulomb force is a piecewise
    4-point cubic whose value jumps slightly where the interval changes; the
    moving M sites sweep thousands of pair distances across such points, so
    finite differences of that term scatter by ~1 % whatever h is.  With the
    tabulated Coulomb term removed (in the oracle and on the device alike)
    every other path of gamma -- PME, excluded-pair correction, ghost
    distribution -- must agree with central differences tightly."""
    import torch

    from piny_b200 import params, system, water
    from piny_b200.lib import DeviceBox
    spec, pos_A = _box()
    pos = pos_A / water.BOHR
    xmod = pos.mean(axis=0)
    th = params.theta_of(spec.model)
    rng = np.random.default_rng(2024)
    tt = th * (1.0 + rng.uniform(-0.02, 0.02, size=th.shape))

    def setup(t):
        S = system.build_system(dataclasses.replace(spec, model=params.model_with(spec.model, t)), pos)
        S["cv0_c"] = S["cv0_c"] * 0.0
        S["cdv0_c"] = S["cdv0_c"] * 0.0
        return S

    S0 = setup(th)
    pi, pj = oracle.verlist(S0, pos[0], xmod, S0["hmat"], S0["cutskin2"])

    def run(t):
        S = setup(t)
        f, e = oracle.energy_force(S, pos, xmod, S["hmat"], pi, pj, distribute_ghosts=True)
        return f, e["vintert"] + e["vintrat"]

    ft, _ = run(tt)
    F, _ = run(th)
    k = params.PARAMS.index("gamma")
    h = 1e-5 * th[k]
    tp, tm = th.copy(), th.copy()
    tp[k] += h
    tm[k] -= h
    (fp, ep), (fm, em) = run(tp), run(tm)
    gL = (((fp - ft) ** 2).sum() - ((fm - ft) ** 2).sum()) / (2 * h)
    gE = (ep - em) / (2 * h)
    box = DeviceBox(S0, spec.nbeads, "fp64")
    box.build_list(pos[0], xmod, S0["hmat"], S0["cutskin2"])
    box.grad_prepare(params.tangents(spec, th, S0))
    d = torch.from_numpy(pos).to("cuda:0")
    dx = torch.from_numpy(xmod).to("cuda:0")
    fb = torch.from_numpy(2.0 * (F - ft)).to("cuda:0")
    dE, dF = box.grad(d.data_ptr(), dx.data_ptr(), S0["hmat"], fb.data_ptr())
    assert abs(dF[k] - gL) <= 1e-7 * abs(gL)
    assert abs(dE[k] - gE) <= 1e-7 * abs(gE)
    box.close()


def test_c5_size_adjoint_matches_device_differences():
    """The gradient configuration itself (1024 q-TIP4P/F, 16 beads, 32^3
    mesh, order 8): the FP64 adjoint against central differences (h = 1e-5
    relative) of the FP64 device energy and force-matching loss, at the
    tolerances above; the MIXED adjoint against the FP64 one."""
    from piny_b200 import params, water
    from piny_b200.params import PARAMS, PinyForceField
    spec = water.named_spec("tip4pf_1024_p16")
    pos_A = water.build_positions(spec)
    theta = params.theta_of(spec.model)
    rng = np.random.default_rng(2024)
    theta_t = theta * (1.0 + rng.uniform(-0.02, 0.02, size=theta.shape))
    field = PinyForceField(spec, pos_A, "fp64")
    _, f_target = field.energy_forces(theta_t)
    gE_fd, gL_fd = np.zeros(len(theta)), np.zeros(len(theta))
    for k in range(len(theta)):
        h = 1e-5 * abs(theta[k])
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        Ep, Fp = field.energy_forces(tp)
        Em, Fm = field.energy_forces(tm)
        gE_fd[k] = (Ep - Em) / (2 * h)
        gL_fd[k] = (((Fp - f_target) ** 2).sum() - ((Fm - f_target) ** 2).sum()) / (2 * h)
    field.close()
    _, _, gE, gL = _adjoint(spec, pos_A, theta, f_target, "fp64")
    sE, sL = np.abs(gE_fd).max(), np.abs(gL_fd).max()
    for k in range(len(theta)):
        assert abs(gE[k] - gE_fd[k]) <= 2e-5 * sE, ("dE", k, gE[k], gE_fd[k])
        assert abs(gL[k] - gL_fd[k]) <= 2e-5 * sL, ("dL", k, gL[k], gL_fd[k])
        if PARAMS[k] != "gamma":
            assert abs(gE[k] - gE_fd[k]) <= 2e-6 * abs(gE_fd[k]), ("dE", PARAMS[k], gE[k], gE_fd[k])
            assert abs(gL[k] - gL_fd[k]) <= 2e-6 * abs(gL_fd[k]), ("dL", PARAMS[k], gL[k], gL_fd[k])
    _, _, gE32, gL32 = _adjoint(spec, pos_A, theta, f_target, "mixed")
    assert np.abs(gE32 - gE).max() <= 1e-3 * np.abs(gE).max()
    assert np.abs(gL32 - gL).max() <= 1e-3 * np.abs(gL).max()
