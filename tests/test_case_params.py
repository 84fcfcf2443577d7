"""Case parameters pinned to the reference's own demo setup scripts
(demo/cavity/para.py, demo/ball/para.py, run by tests/golden/gen_golden.py
into para_golden.json): the gas constant, the density of a Knudsen number,
the dimensionless viscosity and muRef that the case builders use."""
import json
import math
import os

import pytest

from dugks_b200 import case as cs

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "para_golden.json")))


def test_gas_constant_and_demo_values():
    own = GOLD["cavity"]["own"]
    assert cs.K_BOLTZMANN / cs.M_ARGON == pytest.approx(own["R"], rel=1e-15)
    # the demo's DVMProperties and 0/rho carry these with 12 significant digits
    assert cs.R_DEMO == pytest.approx(own["R"], rel=1e-11)
    assert cs.RHO_DEMO == pytest.approx(own["rho"], rel=1e-11)
    assert cs.MU_DEMO == pytest.approx(own["mu"], rel=1e-11)


@pytest.mark.parametrize("kn", ["0.01", "0.075", "0.1", "1.0"])
def test_density_and_viscosity_of_kn(kn):
    for demo, omega in (("cavity", "omega_HS"), ("ball", "omega_VHS")):
        g = GOLD[demo][kn]
        assert cs.rho_from_kn(float(kn), g["L"]) == pytest.approx(g["rho"], rel=1e-15)
        assert cs.mu_bar(float(kn), g[omega]) == pytest.approx(g["muBar"], rel=1e-15)
        assert g["rho"] * g["C"] * g["L"] * g["muBar"] == pytest.approx(g["mu"], rel=1e-15)


@pytest.mark.parametrize("kn", [0.01, 0.1, 1.0])
def test_cavity_density_scales_with_kn(kn):
    c = cs.cavity_case(4, 6, kn=kn)
    assert float(c.rho0[0]) == pytest.approx(GOLD["cavity"][repr(kn)]["rho"], rel=1e-11)


def test_ball_viscosity_follows_the_ball_script():
    """The ball builder takes Kn on the diameter (L = 2) and the ball
    script's VHS viscosity mu = rho C L muBar at the free-stream T."""
    c = cs.ball_case(2, 2, 1.12, 6, kn=0.1, mach=0.5)
    g = GOLD["ball"]["0.1"]
    T = c.gas["Tref"]
    rho = cs.rho_from_kn(0.1, 2.0)
    mu = rho * math.sqrt(2.0 * g["R"] * T) * 2.0 * g["muBar"]
    assert c.gas["muRef"] == pytest.approx(mu, rel=1e-12)
    assert cs.mu_bar(0.1, cs.OMEGA_VHS) == pytest.approx(g["muBar"], rel=1e-15)
