"""DV sets that are no tensor product (the reference's unstructured velocity
mesh, fvDVM.C:129-277): the general-DV passes against the oracle, which
takes any list of velocities and weights.  A tensor-product set given as a
list must give the row-factored path's result; jittered velocity meshes
check the general path itself, in 2-D and 3-D, FP64 and FP32c, with the
boundary types it supports and with DV shards."""
import numpy as np
import pytest

import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import meshgen
from dugks_b200 import quadrature
from dugks_b200 import shard as sh

pytestmark = pytest.mark.gpu


def _vmesh_cavity(n=8, nv=10, jitter=0.2):
    c = cs.cavity_case(n, 8, flatten=False)
    c.use_velocity_mesh(meshgen.velocity_box(nv, 1600.0, 2, jitter=jitter))
    return c.flatten()


def _parity(c, steps, tol=1e-10, floor=1e-4, **kw):
    gpu, orc = dl.Solver(c, **kw), ob.Oracle(c)
    for _ in range(steps):
        gpu.evolution(c.dt)
        orc.evolution(c.dt)
    errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"], floor)
    assert max(errs.values()) <= tol, errs
    return gpu, orc


def test_tensor_set_as_a_list_matches_the_factored_path():
    c = cs.cavity_case(8, 8)
    xi, w = c.dv_set()
    lst = cs.cavity_case(8, 8, flatten=False)
    lst.dv_xi, lst.dv_w = xi, w
    lst.flatten()
    a, b = dl.Solver(c), dl.Solver(lst)
    a.step(6, c.dt)
    b.step(6, lst.dt)
    errs = ob.macro_errors(b.macros(), a.macros(), c.gas["R"])
    assert max(errs.values()) <= 1e-12, errs
    assert ob.rel_l2(b.state()[0], a.state()[0]) <= 1e-12


def test_jittered_velocity_mesh_2d():
    gpu, orc = _parity(_vmesh_cavity(), 8)
    ferrs = ob.macro_errors(gpu.face_macros(), orc.face_macros(), gpu.case.gas["R"])
    assert max(ferrs.values()) <= 1e-10, ferrs
    assert ob.rel_l2(gpu.boundary_rho(), orc.boundary_rho()) <= 1e-10


def test_jittered_velocity_mesh_3d_far_field_ball():
    c = cs.ball_case(4, 4, 1.12, 6, kn=0.1, mach=0.5, flatten=False)
    c.use_velocity_mesh(meshgen.velocity_box(6, 1200.0, 3, jitter=0.15))
    c.flatten()
    _parity(c, 6, tile_cells=32, dv_chunks=3)


def test_velocity_mesh_on_octagon_cells():
    # the general-DV passes on a 2:1 refined cavity: octagons with eight
    # internal faces take their stencil and flux-list fallbacks
    c = cs.refined_cavity_case(6, 8, flatten=False)
    c.use_velocity_mesh(meshgen.velocity_box(8, 1600.0, 2, jitter=0.2))
    c.flatten()
    _parity(c, 8, tile_cells=12, dv_chunks=2)


def test_fp32c_velocity_mesh():
    _parity(_vmesh_cavity(), 8, tol=5e-6, floor=1e-2, precision=dl.FP32C)


def test_velocity_mesh_with_pressure_mixed_and_zero_gradient_patches():
    p1 = cs.R_DEMO * 273.0
    c = cs.channel_case(10, 5, 8, sides={"inlet": {"kind": "pressureIn", "p": 1.2 * p1, "T": 273.0},
                                         "outlet": {"kind": "pressureOut", "p": p1, "T": 273.0},
                                         "top": {"kind": "zeroGradient"},
                                         "bottom": {"kind": "mixed", "rho": 1.0, "U": (30.0, 0.0, 0.0)}},
                        flatten=False)
    c.rho0 = np.full(c.n_cells, 1.0)
    c.use_velocity_mesh(meshgen.velocity_box(10, 1600.0, 2, jitter=0.2))
    c.flatten()
    _parity(c, 8)


def test_velocity_mesh_shards_and_refusals():
    c = _vmesh_cavity()
    shards = [dl.Solver(c, shard=dl.shard(r, 3)) for r in range(3)]
    assert sum(s.n_dv_local for s in shards) == c.n_dv
    sh.step_local(shards, 5, c.dt)
    orc = ob.Oracle(c)
    for _ in range(5):
        orc.evolution(c.dt)
    errs = ob.macro_errors(shards[0].macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= 1e-10, errs
    s = cs.channel_case(6, 3, 6, sides={"top": {"kind": "symmetryPlane"}}, flatten=False)
    s.use_velocity_mesh(meshgen.velocity_box(6, 1600.0, 2))
    s.flatten()
    with pytest.raises(dl.DugksError) as e:
        dl.Solver(s)
    assert e.value.code == 7


# macroFlux yes on a velocity mesh (fvDVM.C:1562-1611): cell rho, rho U,
# rho E advance by the fluxes of the relaxed face DFs
@pytest.mark.parametrize("which", ["cavity", "pressure"])
def test_velocity_mesh_macro_flux(which):
    if which == "cavity":
        c = _vmesh_cavity()
    else:
        p1 = cs.R_DEMO * 273.0
        c = cs.channel_case(10, 5, 8, sides={"inlet": {"kind": "pressureIn", "p": 1.2 * p1, "T": 273.0},
                                             "outlet": {"kind": "pressureOut", "p": p1, "T": 273.0}},
                            flatten=False)
        c.rho0 = np.full(c.n_cells, 1.0)
        c.use_velocity_mesh(meshgen.velocity_box(10, 1600.0, 2, jitter=0.2))
        c.flatten()
    gpu, orc = dl.Solver(c, macro_flux=True), ob.Oracle(c, macro_flux=True)
    for _ in range(8):
        gpu.evolution(c.dt)
        orc.evolution(c.dt)
    errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= 1e-10, errs
    plain = dl.Solver(c)
    plain.step(8, c.dt)
    assert not np.array_equal(plain.macros()["rho"], gpu.macros()["rho"])


# macroFlux yes on a velocity mesh over DV shards: the flux-term moments are
# reduced over the shards together with the cell moments
@pytest.mark.parametrize("world", [2, 3])
def test_velocity_mesh_macro_flux_shards(world):
    c = _vmesh_cavity()
    shards = [dl.Solver(c, macro_flux=True, shard=dl.shard(r, world), dv_chunks=2) for r in range(world)]
    sh.step_local(shards, 6, c.dt)
    plain = dl.Solver(c, macro_flux=True)
    plain.step(6, c.dt)
    orc = ob.Oracle(c, macro_flux=True)
    for _ in range(6):
        orc.evolution(c.dt)
    for s in shards:
        e_plain = ob.macro_errors(s.macros(), plain.macros(), c.gas["R"])
        assert max(e_plain.values()) <= 1e-12, e_plain
        e_orc = ob.macro_errors(s.macros(), orc.macros(), c.gas["R"])
        assert max(e_orc.values()) <= 1e-10, e_orc


def test_velocity_mesh_macro_flux_nccl_one_rank_is_the_unsharded_step():
    c = _vmesh_cavity()
    a = dl.Solver(c, macro_flux=True, shard=dl.shard(0, 1, dl.nccl_unique_id()), dv_chunks=3)
    b = dl.Solver(c, macro_flux=True, dv_chunks=3)
    a.step(5, c.dt)
    b.step(5, c.dt)
    for k in ("rho", "U", "T", "q"):
        assert np.array_equal(a.macros()[k], b.macros()[k]), k
