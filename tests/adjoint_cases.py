"""Cases, objective weights and parameter perturbations shared by the
tangent (oracle) and adjoint (GPU) tests."""
import copy

import numpy as np

from dugks_b200 import case as cs


def objective_weights(c):
    """Energy flux through every boundary face, x-momentum flux through the
    first patch (the lid of the cavity): the wall heat flux and lid shear
    objective.  Returns (energy weights, momentum weights, lid mask)."""
    fl = c.flat
    nb = fl["n_boundary"]
    first = np.zeros(nb, bool)
    first[fl["patch_start"][0]:fl["patch_start"][1]] = True
    fw = np.zeros((nb, 3))
    fw[first, 0] = 1.0
    return np.ones(nb), fw, first


def perturbed(c, eps, dT_b=None, dU_b=None, d_mu=0.0):
    """A copy of case c with T_b += eps dT_b, U_b += eps dU_b, muRef += eps d_mu."""
    cc = copy.copy(c)
    cc.flat = dict(c.flat)
    cc.gas = dict(c.gas)
    if dT_b is not None:
        cc.flat["T_b"] = c.flat["T_b"] + eps * dT_b
    if dU_b is not None:
        cc.flat["U_b"] = c.flat["U_b"] + eps * np.reshape(dU_b, (-1, 3))
    cc.gas["muRef"] = c.gas["muRef"] + eps * d_mu
    return cc


def cases():
    """An 8x8 cavity (walls only) and an 8x4 channel with far-field inlet
    and outlet at other temperatures and a uniform inflow."""
    ff = {"inlet": {"kind": "farField", "T": 300.0}, "outlet": {"kind": "farField", "T": 273.0}}
    ch = cs.channel_case(8, 4, 8, sides=ff, U0=(40.0, 0.0, 0.0), flatten=False)
    rho = float(ch.rho0[0])
    for p in ch.patches:
        if p.kind == "farField":
            p.rho = rho
    return {"cavity": cs.cavity_case(8, 8, kn=0.1), "farfield": ch.flatten()}
