"""The two-phase time step on the device (sipg_ins3d_*) against the composed
oracle step (oracle/ins_oracle.py TwoPhaseStep, whose pieces are pinned against the
reference's kernels in tests/test_ins_oracle.py and tests/test_projection.py), and
the mixed-precision pressure solve against the FP64 one."""
import numpy as np
import pytest

import dg_oracle as D
import ins_oracle as I
import sipg
from helpers import rel_err

pytestmark = pytest.mark.gpu

# the level set's interface width is the reference's default (alpha = 24 h): a factor that
# jumps by 1000 inside one element makes the nodal-factor operator indefinite
CONSTS = dict(reynolds=100.0, rho0=1.0, rho1=1e-3, mu0=1.0, mu1=1e-2, gravity=9.81)


def _case(n, p, open_top, slip_sides=False):
    gm = sipg.Mesh.box(3, n, jitter=0.1, seed=5)
    om = D.Mesh.box(3, n, 0.1, 5)
    t = D.ref_tables(3, p)
    e = om.export(p, t)
    s = np.sqrt((e["x"] - 0.5) ** 2 + (e["y"] - 0.3) ** 2 + (e["z"] - 0.5) ** 2) - 0.25
    # a smooth start that vanishes on the walls, so that advection has work to do
    w = 0.3 * np.sin(np.pi * e["x"]) * np.sin(np.pi * e["y"]) * np.sin(np.pi * e["z"])
    vel = np.stack([w, -0.5 * w, 0.25 * w])
    vel_bc = np.zeros(om.Kb, np.int32)
    if slip_sides:  # slip on the x and z walls, no-slip on the y walls
        c = om.bface_centroid
        vel_bc[(c[:, 1] > 1e-9) & (c[:, 1] < 1.0 - 1e-9)] = I.BC_SLIP
    if open_top:
        vel_bc[om.bface_centroid[:, 1] > 1.0 - 1e-9] = I.BC_OUTFLOW
    return gm, om, s, vel, vel_bc


def _mean_free(p):
    return p - p.mean()


@pytest.mark.parametrize("p", [2, 3])
@pytest.mark.parametrize("open_top", [False, True], ids=["closed", "open-top"])
def test_two_phase_steps_match_the_oracle(p, open_top):
    gm, om, s, vel, vel_bc = _case(3, p, open_top)
    tol = dict(pr_rel_tol=1e-11, pr_abs_tol=1e-300, vis_rel_tol=1e-11, vis_abs_tol=1e-300)
    ins = sipg.Ins3D(gm, vel_bc, order=p, precision=sipg.FP64, **tol, **CONSTS)
    ins.set_state(vel, s)
    ref = I.TwoPhaseStep(om, p, vel_bc, **CONSTS)
    ref.set_state(vel, s)
    for k in range(3):
        info = ins.step()
        ref.step()
        assert info.proj_converged == gm.K
        assert info.time == pytest.approx(ref.time, rel=1e-12)
        assert info.dt == pytest.approx(ref.dt, rel=1e-9)
    got = ins.state()
    # solves stop at 1e-11 relative residual on both sides
    assert rel_err(got["vel"], ref.vel) < 1e-7
    assert rel_err(got["s"], ref.s) < 1e-9
    pg, pw = (got["pr"], ref.pr) if open_top else (_mean_free(got["pr"]), _mean_free(ref.pr))
    assert rel_err(pg, pw) < 1e-7
    assert rel_err(got["rho"], ref.rho) < 1e-9 and rel_err(got["mu"], ref.mu) < 1e-9


def test_mixed_pressure_preconditioner_steps_match_fp64():
    """The time step with the FP32 p-multigrid V-cycle inside the FP64 outer Krylov
    solve against the all-FP64 one, both at the reference's tolerances."""
    gm, _, s, vel, vel_bc = _case(4, 3, False)
    runs = {}
    for prec in (sipg.FP64, sipg.FP32):
        ins = sipg.Ins3D(gm, vel_bc, order=3, precision=prec, **CONSTS)
        ins.set_state(vel, s)
        infos = [ins.step() for _ in range(4)]
        runs[prec] = (ins.state(), infos)
    a, b = runs[sipg.FP64][0], runs[sipg.FP32][0]
    assert rel_err(b["vel"], a["vel"]) < 1e-5
    assert rel_err(b["s"], a["s"]) < 1e-7
    for i64, i32 in zip(runs[sipg.FP64][1], runs[sipg.FP32][1]):
        assert abs(i64.pr_iters - i32.pr_iters) <= 2


def test_over_integrated_pressure_equals_nodal_for_one_density():
    """One density: the factor is 1 at every cubature point and the over-integrated
    operator is the nodal one, so the steps agree to the solver tolerance."""
    gm, _, s, vel, vel_bc = _case(3, 2, False)
    consts = dict(CONSTS, rho1=1.0)
    tol = dict(pr_rel_tol=1e-11, pr_abs_tol=1e-300, vis_rel_tol=1e-11, vis_abs_tol=1e-300)
    got = []
    for over_int in (0, 1):
        ins = sipg.Ins3D(gm, vel_bc, order=2, precision=sipg.FP64, pr_over_int=over_int, **tol, **consts)
        ins.set_state(vel, s)
        ins.step(3)
        got.append(ins.state())
    assert rel_err(got[1]["vel"], got[0]["vel"]) < 1e-8
    assert rel_err(_mean_free(got[1]["pr"]), _mean_free(got[0]["pr"])) < 1e-8


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "mixed"])
def test_over_integrated_two_phase_steps_converge_and_lift_the_bubble(precision):
    gm, _, s, vel, vel_bc = _case(4, 3, False)
    vel[:] = 0.0
    ins = sipg.Ins3D(gm, vel_bc, order=3, precision=precision, pr_over_int=1, **CONSTS)
    ins.set_state(vel, s)
    for _ in range(4):
        info = ins.step()
        assert info.pr_iters < 500 and info.pr_rel_res <= 1e-8
    st = ins.state()
    assert st["vel"][1][s < 0].mean() > 0


def test_block_jacobi_viscous_solves_give_the_jacobi_steps():
    """[viscous-solve] preconditioner = block-jacobi: the same step to the solver tolerance."""
    gm, _, s, vel, vel_bc = _case(3, 2, False)
    tol = dict(pr_rel_tol=1e-11, pr_abs_tol=1e-300, vis_rel_tol=1e-11, vis_abs_tol=1e-300)
    got, iters = [], []
    for vk in (sipg.SOLVER_JACOBI, sipg.SOLVER_BLOCK_JACOBI):
        ins = sipg.Ins3D(gm, vel_bc, order=2, precision=sipg.FP64, viscous_kind=vk, **tol, **CONSTS)
        ins.set_state(vel, s)
        info = ins.step(2)
        got.append(ins.state())
        iters.append(sum(info.vis_iters))
    assert rel_err(got[1]["vel"], got[0]["vel"]) < 1e-8
    assert iters[1] < iters[0]


@pytest.mark.parametrize("slip", [False, True], ids=["no-slip", "slip-sides"])
def test_inner_fp32_pcg_viscous_solves_give_the_jacobi_steps(slip):
    """viscous_kind = p-multigrid with n_levels 0: the FP64 flexible PCG preconditioned by
    six FP32 Jacobi-PCG iterations on the viscous operator reaches the Jacobi solve's
    steps to the solver tolerance, in far fewer outer iterations; with slip side walls
    through the coupled vector operator."""
    gm, _, s, vel, vel_bc = _case(3, 2, False, slip_sides=slip)
    tol = dict(pr_rel_tol=1e-11, pr_abs_tol=1e-300, vis_rel_tol=1e-11, vis_abs_tol=1e-300)
    inner = dict(viscous_kind=sipg.SOLVER_PMULTIGRID, vis_precision=sipg.FP32, vis_n_levels=0, vis_coarse_iters=6)
    got, iters = [], []
    for kw in ({}, inner):
        ins = sipg.Ins3D(gm, vel_bc, order=2, precision=sipg.FP64, **kw, **tol, **CONSTS)
        ins.set_state(vel, s)
        info = ins.step(2)
        assert all(r <= 1e-11 for r in info.vis_rel_res[:(1 if slip else 3)])
        got.append(ins.state())
        iters.append(sum(info.vis_iters))
        ins.close()
    assert rel_err(got[1]["vel"], got[0]["vel"]) < 1e-8
    assert 2 * iters[1] < iters[0]


@pytest.mark.parametrize("open_top", [False, True], ids=["closed", "open-top"])
def test_over_integrated_two_phase_steps_match_the_oracle(open_top):
    """[pressure-solve] over_int = 1: 1/rho at the cubature points from the level set and
    the over-integrated operator in the pressure solve, against the oracle's step with
    its over-integrated operator (oracle/oi_oracle.py) as the solve's operator."""
    gm, om, s, vel, vel_bc = _case(3, 2, open_top)
    tol = dict(pr_rel_tol=1e-11, pr_abs_tol=1e-300, vis_rel_tol=1e-11, vis_abs_tol=1e-300)
    ins = sipg.Ins3D(gm, vel_bc, order=2, precision=sipg.FP64, pr_over_int=1, **tol, **CONSTS)
    ins.set_state(vel, s)
    ref = I.TwoPhaseStep(om, 2, vel_bc, over_int=True, **CONSTS)
    ref.set_state(vel, s)
    for _ in range(2):
        ins.step()
        ref.step()
    got = ins.state()
    assert rel_err(got["vel"], ref.vel) < 1e-7
    pg, pw = (got["pr"], ref.pr) if open_top else (_mean_free(got["pr"]), _mean_free(ref.pr))
    assert rel_err(pg, pw) < 1e-7


@pytest.mark.parametrize("open_top", [False, True], ids=["closed", "open-top"])
def test_slip_walls_two_phase_steps_match_the_oracle(open_top):
    """Slip side walls: the coupled vector viscous solve (uses_slip_bcs) in the driver
    against the oracle's vector solve on the same operator."""
    gm, om, s, vel, vel_bc = _case(3, 2, open_top, slip_sides=True)
    tol = dict(pr_rel_tol=1e-11, pr_abs_tol=1e-300, vis_rel_tol=1e-11, vis_abs_tol=1e-300)
    ins = sipg.Ins3D(gm, vel_bc, order=2, precision=sipg.FP64, **tol, **CONSTS)
    ins.set_state(vel, s)
    ref = I.TwoPhaseStep(om, 2, vel_bc, **CONSTS)
    ref.set_state(vel, s)
    for _ in range(3):
        info = ins.step()
        ref.step()
        assert info.vis_iters[0] == info.vis_iters[1] == info.vis_iters[2] > 0
    got = ins.state()
    assert rel_err(got["vel"], ref.vel) < 1e-7
    assert rel_err(got["s"], ref.s) < 1e-9


@pytest.mark.parametrize("over_int", [0, 1], ids=["nodal", "over-integrated"])
def test_lagged_pressure_setup_gives_the_same_steps(over_int):
    """pr_setup_every = 3: the V-cycle set up every third step only; the solves still reach
    their tolerance, so the steps agree with the every-step set-up."""
    gm, _, s, vel, vel_bc = _case(3, 2, False)
    tol = dict(pr_rel_tol=1e-11, pr_abs_tol=1e-300, vis_rel_tol=1e-11, vis_abs_tol=1e-300)
    got, iters = [], []
    for every in (1, 3):
        ins = sipg.Ins3D(gm, vel_bc, order=2, precision=sipg.FP32, pr_over_int=over_int, pr_setup_every=every,
                         **tol, **CONSTS)
        ins.set_state(vel, s)
        its = [ins.step().pr_iters for _ in range(5)]
        got.append(ins.state())
        iters.append(its)
    assert rel_err(got[1]["vel"], got[0]["vel"]) < 1e-7
    assert max(iters[1]) <= 2 * max(iters[0]) + 5
