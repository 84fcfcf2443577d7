"""The standalone C++ host (psp-vst_b200/host: FoamFile reader, FvDVM over
the C ABI, dugks_run driver) against the Python host path on the same case
files.  Without a GPU: the case reader and the mesh flattening
(`dugks_run --check`).  With a GPU: steps through the driver give the same
fields as the Python Solver."""
import json
import os
import subprocess

import numpy as np
import pytest

import case_writer
import golden_cases
from dugks_b200 import case as cs
from dugks_b200 import foamio
from dugks_b200 import lib as dl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "psp-vst_b200", "host")
DRIVER = os.path.join(HOST, "bin", "dugks_run")


@pytest.fixture(scope="module")
def driver():
    dl.load()   # the library the driver links
    subprocess.run(["make", "-s", "-C", HOST], check=True)
    assert os.path.exists(DRIVER)
    return DRIVER


def _run(driver, *args, check=True):
    r = subprocess.run([driver, *map(str, args)], capture_output=True, text=True, timeout=600)
    if check:
        assert r.returncode == 0, r.stderr
    return r


def _summary(r) -> dict:
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_check_demo_cavity(driver, tmp_path):
    c = golden_cases.demo_cavity()
    d = case_writer.write_case(c, str(tmp_path / "cavity"))
    s = _summary(_run(driver, d, "--check"))
    fl = c.flat
    assert s["cells"] == c.n_cells == 3600
    assert s["internal_faces"] == fl["n_internal"] and s["boundary_faces"] == fl["n_boundary"] == 240
    assert s["D"] == 2 and s["n_dv"] == 28 ** 2
    assert s["volume"] == pytest.approx(float(np.sum(fl["V"])), rel=1e-14)
    assert s["mass"] == pytest.approx(float(np.sum(c.rho0 * fl["V"])), rel=1e-14)
    assert s["xi_max"] == c.xi_max
    kinds = {p["name"]: p["kind"] for p in s["patches"]}
    assert kinds == {"movingWall": "maxwellWall", "fixedWalls": "maxwellWall", "frontAndBack": "empty"}


def test_check_ball_far_field(driver, tmp_path):
    c = cs.ball_case(4, 4, 1.12, 6, kn=0.1, mach=0.5)
    d = case_writer.write_case(c, str(tmp_path / "ball"))
    s = _summary(_run(driver, d, "--check"))
    assert s["cells"] == c.n_cells and s["D"] == 3 and s["n_dv"] == 216
    assert s["boundary_faces"] == c.flat["n_boundary"]
    kinds = {p["name"]: p["kind"] for p in s["patches"]}
    assert kinds == {"wall": "maxwellWall", "farField": "farField"}
    assert s["volume"] == pytest.approx(float(np.sum(c.flat["V"])), rel=1e-14)


def test_check_reads_time_controls(driver, tmp_path):
    # readTimeControlsExplicit.H: adjustTimeStep (a Switch), maxCo, maxDeltaT
    c = cs.cavity_case(4, 6)
    d = case_writer.write_case(c, str(tmp_path / "a"), control={"deltaT": 1e-5, "adjustTimeStep": "on",
                                                                "maxCo": 0.7, "maxDeltaT": 2e-5})
    s = _summary(_run(driver, d, "--check"))
    assert s["adjust_time_step"] is True and s["max_co"] == 0.7 and s["max_delta_t"] == 2e-5
    d = case_writer.write_case(c, str(tmp_path / "b"), control={"deltaT": 1e-5})
    s = _summary(_run(driver, d, "--check"))
    assert s["adjust_time_step"] is False and s["max_co"] == 1.0 and s["max_delta_t"] == 1e15
    d = case_writer.write_case(c, str(tmp_path / "c"), control={"adjustTimeStep": "maybe"})
    r = _run(driver, d, "--check", check=False)
    assert r.returncode == 1 and "maybe" in r.stderr


def test_unsupported_patch_type_is_an_error(driver, tmp_path):
    c = cs.cavity_case(4, 6)
    d = case_writer.write_case(c, str(tmp_path / "bad"), rho_patch_type={"movingWall": "inletOutlet"})
    r = _run(driver, d, "--check", check=False)
    assert r.returncode == 1 and "inletOutlet" in r.stderr


def test_missing_case_is_an_error(driver, tmp_path):
    r = _run(driver, str(tmp_path / "nothing"), "--check", check=False)
    assert r.returncode == 1 and "cannot open" in r.stderr


@pytest.mark.gpu
def test_driver_steps_match_python_solver(driver, tmp_path):
    c = golden_cases.demo_cavity()
    d = case_writer.write_case(c, str(tmp_path / "cavity"))
    steps = 3
    s = _summary(_run(driver, d, "--steps", steps, "--dt", repr(c.dt)))
    assert s["steps"] == steps and s["dt"] == c.dt
    ref = dl.Solver(c)
    ref.step(steps, c.dt)
    m = ref.macros()
    sizes = {p["name"]: p["nFaces"] for p in c.mesh.patches}
    tdir = os.path.join(d, s["time_name"])
    rho = foamio.read_vol_field(os.path.join(tdir, "rho"), c.n_cells, sizes)
    U = foamio.read_vol_field(os.path.join(tdir, "U"), c.n_cells, sizes)
    T = foamio.read_vol_field(os.path.join(tdir, "T"), c.n_cells, sizes)
    q = foamio.read_vol_field(os.path.join(tdir, "q"), c.n_cells, sizes)
    # the fields are written with 15 significant digits
    np.testing.assert_allclose(rho["internal"], m["rho"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(T["internal"], m["T"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(U["internal"], m["U"], rtol=1e-14, atol=1e-14 * np.abs(m["U"]).max())
    np.testing.assert_allclose(q["internal"], m["q"], rtol=1e-14, atol=1e-14 * np.abs(m["q"]).max())
    assert rho["patches"]["movingWall"]["type"] == "calculatedMaxwell"
    np.testing.assert_allclose(rho["patches"]["movingWall"]["value"],
                               ref.boundary_rho()[: sizes["movingWall"]], rtol=1e-14)
    assert s["mass"] == pytest.approx(float(np.sum(m["rho"] * c.flat["V"])), rel=1e-13)


@pytest.mark.gpu
def test_restart_file_continues_exactly(driver, tmp_path):
    # 4 steps straight vs 2 steps, an exact restart file, then 2 more steps:
    # the written fields are identical, byte for byte
    c = cs.cavity_case(12, 8)
    a = case_writer.write_case(c, str(tmp_path / "straight"))
    b = case_writer.write_case(c, str(tmp_path / "restarted"))
    sa = _summary(_run(driver, a, "--steps", 4, "--dt", repr(c.dt)))
    s1 = _summary(_run(driver, b, "--steps", 2, "--dt", repr(c.dt), "--write-state"))
    header, dfs = 8 + 4 + 4 + 8 + 8 + 8 + 8, 2 * 8 * c.n_cells * 64
    record = 8 * (9 * c.n_cells + 2 + 2 * c.flat["n_boundary"])
    assert os.path.getsize(os.path.join(b, s1["time_name"], "dugksState")) == header + dfs + record
    sb = _summary(_run(driver, b, "--steps", 2, "--dt", repr(c.dt), "--restart", s1["time_name"]))
    assert sa["time_name"] == sb["time_name"]
    for name in ("rho", "U", "T", "q"):
        with open(os.path.join(a, sa["time_name"], name)) as fa, open(os.path.join(b, sb["time_name"], name)) as fb:
            assert fa.read() == fb.read(), name


@pytest.mark.gpu
def test_restart_rejects_another_mesh(driver, tmp_path):
    c = cs.cavity_case(12, 8)
    b = case_writer.write_case(c, str(tmp_path / "one"))
    s1 = _summary(_run(driver, b, "--steps", 1, "--dt", repr(c.dt), "--write-state"))
    other = case_writer.write_case(cs.cavity_case(10, 8), str(tmp_path / "two"))
    os.makedirs(os.path.join(other, s1["time_name"]))
    os.replace(os.path.join(b, s1["time_name"], "dugksState"), os.path.join(other, s1["time_name"], "dugksState"))
    r = _run(driver, other, "--steps", 1, "--dt", repr(c.dt), "--restart", s1["time_name"], check=False)
    assert r.returncode == 1 and "another mesh" in r.stderr


@pytest.mark.gpu
def test_adjustable_time_step_from_control_dict(driver, tmp_path):
    # adjustTimeStep yes: each step runs CourantNo.H + setDeltaTvar.H on the
    # device; the driver's steps equal Solver.step_adaptive's, and the run
    # stops at endTime as Time::run does
    c = cs.cavity_case(12, 8)
    dt0 = 0.3 * c.dt
    end = 6.0 * c.dt
    control = {"startTime": 0.0, "endTime": end, "deltaT": dt0, "writeInterval": 1.0,
               "adjustTimeStep": "yes", "maxCo": 0.5}
    d = case_writer.write_case(c, str(tmp_path / "adjust"), control=control)
    s = _summary(_run(driver, d))
    ref = dl.Solver(c)
    t, dt, n = 0.0, dt0, 0
    while t < end - 0.5 * dt:
        dt, _ = ref.step_adaptive(1, dt, 0.5, 1e15)
        t += dt
        n += 1
    assert s["steps"] == n and s["dt"] == dt and s["time"] == t
    m = ref.macros()
    sizes = {p["name"]: p["nFaces"] for p in c.mesh.patches}
    rho = foamio.read_vol_field(os.path.join(d, s["time_name"], "rho"), c.n_cells, sizes)
    np.testing.assert_allclose(rho["internal"], m["rho"], rtol=1e-14, atol=0)


def _channel_sides():
    p = 1.0 * cs.R_DEMO * 273.0
    return {"inlet": {"kind": "pressureIn", "p": 1.2 * p, "T": 273.0},
            "outlet": {"kind": "pressureOut", "p": p, "T": 273.0},
            "bottom": {"kind": "zeroGradient"}, "top": {"kind": "symmetryPlane"}}


def test_check_reads_every_rho_patch_type(driver, tmp_path):
    kinds = {"inlet": "mixed", "outlet": "zeroGradient", "bottom": "DVMsymmetry", "top": "farField"}
    c = cs.channel_case(6, 3, 6, sides={k: {"kind": v, "rho": 1e-6} for k, v in kinds.items()})
    d = case_writer.write_case(c, str(tmp_path / "a"))
    s = _summary(_run(driver, d, "--check"))
    got = {p["name"]: p["kind"] for p in s["patches"]}
    assert got == dict(kinds, frontAndBack="empty")
    c = cs.channel_case(6, 3, 6, sides=_channel_sides())
    d = case_writer.write_case(c, str(tmp_path / "b"))
    got = {p["name"]: p["kind"] for p in _summary(_run(driver, d, "--check"))["patches"]}
    assert got == {"inlet": "pressureIn", "outlet": "pressureOut", "bottom": "zeroGradient", "top": "symmetryPlane",
                   "frontAndBack": "empty"}


@pytest.mark.gpu
def test_driver_pressure_driven_channel_matches_python_solver(driver, tmp_path):
    c = cs.channel_case(12, 6, 8, sides=_channel_sides(), flatten=False)
    c.rho0 = np.full(c.n_cells, 1.0)
    c.flatten()
    d = case_writer.write_case(c, str(tmp_path / "channel"))
    s = _summary(_run(driver, d, "--steps", 6, "--dt", repr(c.dt)))
    ref = dl.Solver(c)
    ref.step(6, c.dt)
    m = ref.macros()
    sizes = {p["name"]: p["nFaces"] for p in c.mesh.patches}
    rho = foamio.read_vol_field(os.path.join(d, s["time_name"], "rho"), c.n_cells, sizes)
    np.testing.assert_allclose(rho["internal"], m["rho"], rtol=1e-14, atol=0)


def test_check_reads_macro_flux(driver, tmp_path):
    c = cs.cavity_case(4, 6)
    c.macro_flux = True
    d = case_writer.write_case(c, str(tmp_path / "mf"))
    assert _summary(_run(driver, d, "--check"))["macro_flux"] is True
    c.macro_flux = False
    d = case_writer.write_case(c, str(tmp_path / "nomf"))
    assert _summary(_run(driver, d, "--check"))["macro_flux"] is False


def _vmesh_case():
    from dugks_b200 import meshgen
    c = cs.cavity_case(6, 6, flatten=False)
    c.use_velocity_mesh(meshgen.velocity_box(8, 1600.0, 2, jitter=0.2))
    return c.flatten()


def test_check_reads_the_velocity_mesh(driver, tmp_path):
    c = _vmesh_case()
    d = case_writer.write_case(c, str(tmp_path / "vm"))
    s = _summary(_run(driver, d, "--check", "--vmesh"))
    assert s["n_dv"] == 64 and s["xi_max"] == pytest.approx(c.xi_max, rel=1e-14)
    assert _summary(_run(driver, d, "--check"))["n_dv"] == 36      # 6^2 from Xis without --vmesh


@pytest.mark.gpu
def test_driver_velocity_mesh_matches_python_solver(driver, tmp_path):
    c = _vmesh_case()
    d = case_writer.write_case(c, str(tmp_path / "vm"))
    s = _summary(_run(driver, d, "--vmesh", "--steps", 4, "--dt", repr(c.dt)))
    assert s["n_dv"] == 64
    ref = dl.Solver(c)
    ref.step(4, c.dt)
    sizes = {p["name"]: p["nFaces"] for p in c.mesh.patches}
    rho = foamio.read_vol_field(os.path.join(d, s["time_name"], "rho"), c.n_cells, sizes)
    np.testing.assert_allclose(rho["internal"], ref.macros()["rho"], rtol=1e-13, atol=0)
