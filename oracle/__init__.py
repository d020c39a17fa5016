"""CPU oracle for the DG Euler/Navier-Stokes right-hand side.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this package, and only as the
checker (or as the timed CPU restatement of the reference).  The product path
in ``mirgecom_b200`` never imports it.

The oracle restates, in float64 numpy, the algorithm of the reference's
array-context path (mirgecom/euler.py, navierstokes.py, operators.py,
inviscid.py, viscous.py, flux.py, gas_model.py, eos.py, transport.py,
thermochemistry.py, boundary.py, integrators/explicit_rk.py), one numpy
operation per reference operation, element-batched.

Parity status: the reference cannot be imported or run here (its runtime --
grudge, meshmode, modepy, pyopencl, pyrometheus, cantera -- is absent), so
agreement with the reference's own numbers is pinned only through the
reference's analytic tests restated in ``tests/`` (uniform state gives a zero
RHS, isentropic-vortex and gradient convergence orders, hand-computed flux
values) and, for thermochemistry, through identities (e(T(e)) round trip, mass
conservation of the source terms, detailed balance).  Bit-level agreement with
grudge's node ordering and matrices is unpinned.
"""
