"""CPU oracle for the RBM variational-Monte-Carlo step of QES (pyqusolver).

TEST INFRASTRUCTURE ONLY.  This package is a float64 NumPy restatement of the
reference algorithm.  It is imported only by ``tests/``, by
``__graft_entry__.smoke()`` (as the checker) and by ``bench.py`` (the
``cpu_baseline`` leg and ``--impl reference``).  The product package
``pyqusolver_b200`` never imports it: its compute path is the CUDA library and
it raises when that library is missing.

The reference (``Python/QES``) is pure Python/JAX and its arithmetic core lives
in the ``general_python`` git submodule, which is empty in the reference
snapshot (RBM, ratio estimator, SR solvers, lattices).  Where the submodule
holds the algorithm, the restatement follows the reference's call sites and
tests, and every unpinned convention is named in the module that makes it:

* ``philox``      -- Philox4x32-10 counter RNG (Salmon et al., SC'11), pinned
                     by published known-answer vectors.
* ``lattice``     -- square/chain lattice, forward bonds, neighbour table
                     (``QES/Solver/MonteCarlo/updates/utils.py:37-109``).
* ``hamiltonian`` -- TFIM / XXZ / J1-J2 term lists and the connected-state
                     enumeration (``QES/Algebra/Hamil/hamil_energy_jax.py:428-576``).
* ``rbm``         -- RBM log-amplitude, theta cache, fast ratio, log-derivatives.
* ``estimator``   -- local energy by full re-evaluation of every connected state
                     (the reference's ``apply_callable_batched_jax`` contract).
* ``sampler``     -- Metropolis chains with the reference's schedule semantics
                     (``QES/Solver/MonteCarlo/vmc.py:952-1283``).
* ``sr``          -- stochastic reconfiguration / TDVP solve
                     (``QES/NQS/src/tdvp.py:1056-1422``).
* ``ed``          -- exact ground-state energy with SciPy ``eigsh``.
* ``vmc``         -- one whole VMC step (sample, E_loc, O, SR, update).
"""
