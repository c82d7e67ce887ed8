"""The two-phase driver's host side (no GPU needed): the option defaults are the
reference's, and bad arguments are refused before any device work."""
import ctypes as C

import numpy as np
import pytest

import sipg


def test_default_options_are_the_references():
    o = sipg.ins3d_default_opts()
    # setup_pressure_viscous_solvers (src/solvers/3d/ins_solver_base.cpp:149-184)
    assert (o.pressure.rel_tol, o.pressure.abs_tol, o.pressure.max_iter) == (1e-8, 1e-9, 500)
    assert (o.viscous.rel_tol, o.viscous.abs_tol, o.viscous.max_iter) == (1e-8, 1e-9, 5000)
    # eigen_val_saftey_factor of the 3D two-phase examples, level-set options, LS_CAP
    assert o.pressure.eig_safety == 2.5
    assert (o.ls_alpha, o.reinit_freq, o.reinit_ic, o.ls_cap) == (24.0, 24, 1, 1.0)
    assert o.viscous_kind == sipg.SOLVER_JACOBI and o.pr_over_int == 0 and o.gravity == 0.0
    assert o.pressure.precision == sipg.FP64 and o.extrapolate_history == 3


def test_option_overrides_reach_the_solver_options():
    o = sipg.ins3d_default_opts(precision=sipg.FP32, pr_cheb_order=6, vis_max_iter=7, reinit_freq=0)
    assert o.pressure.precision == sipg.FP32 and o.pressure.cheb_order == 6
    assert o.viscous.max_iter == 7 and o.reinit_freq == 0


@pytest.mark.parametrize("bad", [dict(reynolds=0.0), dict(rho1=-1.0), dict(ls_cap=0.0), dict(order=5),
                                 dict(viscous_kind=sipg.SOLVER_CG), dict(extrapolate_history=9)])
def test_bad_options_are_refused(bad):
    mesh = sipg.Mesh.box(3, 2, jitter=0.1, seed=1)
    o = sipg.ins3d_default_opts(**bad)
    h = C.c_void_p()
    bc = np.zeros(mesh.Kb, np.int32)
    st = sipg.lib().sipg_ins3d_create(mesh.h, C.byref(o), bc.ctypes.data_as(C.c_void_p), C.byref(h))
    assert st == sipg.SIPG_INVALID_ARG and not h.value


@pytest.mark.parametrize("kind", [sipg.SOLVER_JACOBI, sipg.SOLVER_BLOCK_JACOBI, sipg.SOLVER_PMULTIGRID])
def test_viscous_kinds_the_driver_takes_pass_the_option_checks(kind):
    """Jacobi, block-Jacobi and the FP32 inner Jacobi-PCG preconditioner (p-multigrid
    kind with n_levels 0) get past the option checks; without a GPU the creation then
    stops at the first device call, with a CUDA status rather than SIPG_INVALID_ARG."""
    mesh = sipg.Mesh.box(3, 2, jitter=0.1, seed=1)
    o = sipg.ins3d_default_opts(viscous_kind=kind, vis_precision=sipg.FP32, vis_n_levels=0, vis_coarse_iters=6)
    h = C.c_void_p()
    bc = np.zeros(mesh.Kb, np.int32)
    st = sipg.lib().sipg_ins3d_create(mesh.h, C.byref(o), bc.ctypes.data_as(C.c_void_p), C.byref(h))
    if h.value:
        sipg.lib().sipg_ins3d_destroy(h)
    assert st != sipg.SIPG_INVALID_ARG


def test_unknown_boundary_types_are_refused():
    mesh = sipg.Mesh.box(3, 2, jitter=0.1, seed=1)
    bc = np.full(mesh.Kb, 3, np.int32)  # a custom type of problem_specific_3d.h
    with pytest.raises(sipg.SipgError, match="no-slip"):
        sipg.Ins3D(mesh, bc)


def test_geometry_precision_is_16_or_32_bits():
    mesh = sipg.Mesh.box(3, 2, jitter=0.1, seed=1)
    mesh.set_geometry_precision(16)
    mesh.set_geometry_precision(32)
    with pytest.raises(sipg.SipgError, match="16 or 32"):
        mesh.set_geometry_precision(8)
