"""Golden fixture of the reference's hybrid solver with the 11 Air-11 species carried as extra
conserved variables (16 per node), made by running the reference's own code.

    python tests/golden/make_golden_species.py [/path/to/reference]

Same machinery and outputs as ``make_golden.py`` (``run_case``: metrics, residuals, dt, limiter,
troubled flags, checked steps, the MOOD subcell recompute and MOOD step) on the 3x3x2 jittered
hexahedron box at P2, with smooth and shocked states whose mass fractions vary in space.
Writes ``tests/golden/species_p2.npz``.
"""

import numpy as np

import make_golden as mg

SPECIES = ("e-", "N+", "O+", "NO+", "N2+", "O2+", "N", "O", "NO", "N2", "O2")
_flow = mg.smooth_primitive


def smooth_with_species(xyz):
    """The flow of make_golden.smooth_primitive and mass fractions [e-, N+, O+, NO+, N2+, O2+, N,
    O, NO, N2, O2] that follow its density (the shocked state reuses them)."""
    W = _flow(xyz)
    s = 0.5 + 0.5 * np.tanh(4.0 * (W[..., 0] - 1.0))
    Y = np.zeros(W.shape[:-1] + (11,))
    Y[..., 6] = 0.01 * s
    Y[..., 7] = 0.03 * s
    Y[..., 8] = 0.02 * s
    Y[..., 10] = 0.233 - 0.045 * s
    Y[..., 9] = 1.0 - Y.sum(axis=-1)
    return np.concatenate([W, Y], axis=-1)


def main():
    mg.smooth_primitive = smooth_with_species
    ff = [1.0, 0.6, 0.1, 0.0, 1.0] + [0.0] * 9 + [0.767, 0.233]
    box = mg.meshgen.box_hex((3, 3, 2), lo=(0, 0, 0), hi=(1.5, 1.5, 1.0), jitter=0.15, seed=7)
    mg.run_case("species_p2", box, 2, 0.01, ff, 1.2, 0.6, mood=True, species=SPECIES)


if __name__ == "__main__":
    main()
