"""Directional derivatives of the FP64 CPU oracle's GW self-energy at the differentiable-step size
(nk=27 (3x3x3), nao=20, naux=100, ns=1, ntau=80, beta=100, generator seed 0), for checking the GPU
adjoint at that size without running the oracle on the GPU machine.

For the cotangent Sb (seed 7) and directions E_G (seed 9) in G and E_V (seed 8) in the half-stored
integrals, writes c4_directional.json with the central differences (step 1e-6) of
L = Re sum conj(Sb) Sigma(G, V) along each direction.  The GPU test compares Re<Gb, E_G> and
Re<Vb, E_V> from gb200_gw_sigma_vjp with them.

    python tests/golden/make_c4_directional.py      (about 4 minutes on 8 cores)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, ".."))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, "..", "..", "green-mbpt_b200"))

import gw_oracle as O  # noqa: E402
from gb200 import synth  # noqa: E402

SEED_SB, SEED_EG, SEED_EV, H = 7, 9, 8, 1e-6


def cotangent(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def main():
    s = synth.make_config("c4", seed=0)
    g = s.grid
    bz = O.NoSymBZ(s.mesh)
    Sb = cotangent(s.G.shape, SEED_SB)
    EG = cotangent(s.G.shape, SEED_EG)
    EV = cotangent(s.V_half.shape, SEED_EV)

    def loss(G, V):
        Sig = O.gw_solve(G, O.HalfStoredIntegrals(V), bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ)
        return float(np.real(np.vdot(Sb, Sig)))

    fd_G = (loss(s.G + H * EG, s.V_half) - loss(s.G - H * EG, s.V_half)) / (2 * H)
    fd_V = (loss(s.G, s.V_half + H * EV) - loss(s.G, s.V_half - H * EV)) / (2 * H)
    out = {"config": "c4", "generator_seed": 0, "seed_cotangent": SEED_SB, "seed_dir_G": SEED_EG,
           "seed_dir_V": SEED_EV, "step": H, "fd_G": fd_G, "fd_V": fd_V}
    with open(os.path.join(HERE, "c4_directional.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
