"""CPU oracle for the StoPEPS sample-ensemble hot path.

TEST INFRASTRUCTURE ONLY: the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
anything from this package.  It is a NumPy FP64 restatement of the
reference's Julia files cited in each module (``z2``, ``model``,
``boundary``, ``diagonal``, ``variational``, ``diagonal_variational``,
``full_update``, ``sampling``, ``driver``, and ``adjoint``: the reverse-mode
derivative of lognorm, which the reference does not have).

Parity status: the reference (pure Julia over TensorKit/MatrixAlgebraKit,
neither installed here) ships no golden vectors and cannot be run in this
container, so the oracle is pinned only by exact diagonalization
(``model.exact_thermal_observables``, restating ``src/models/tfim.jl:72-76``)
and by structural invariants.  Parity with the reference itself is
unpinned.
"""
