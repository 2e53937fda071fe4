"""CPU oracle for the hybrid-mesh DG residual-and-update path.

TEST INFRASTRUCTURE ONLY.  This package restates, in plain numpy/float64, the
algorithm of superboss2300/jax-fluid-sim's ``hybrid/`` solver (reference
elements, face pairing, isoparametric metrics, HLLC/Rusanov fluxes, the
anchor-form Euler residual, BR2 viscous residual, SSP-RK3 with positivity and
MOOD subcell FV, Air-11 chemistry).  Every function cites the reference
``file:line`` it follows.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import it, and only as the checker or the timed CPU baseline.  The
product path (``jax_fluid_sim_b200``) never imports it.

Parity of this restatement is pinned against fixtures produced by running the
reference's own Python (under a numpy stand-in for JAX, in the build
container) -- see ``tests/golden/make_golden.py`` and ``tests/test_oracle_golden.py``.
One documented extension: periodic face pairing (the reference hybrid mesh has
none), used by the Taylor-Green and vortex workloads.
"""
