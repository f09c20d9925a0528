"""CPU oracle for the FETI dual-iteration hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library imports, links or
executes this package; it is used exclusively by ``tests/``, by
``__graft_entry__.smoke()`` as the checker, and by ``bench.py``'s CPU
baseline leg.  It is a plain numpy/scipy restatement of ESPRESO's
(feeleewee/espreso) Total-FETI algorithm:

* ``oracle.mesh``       -- grid generator, HEXA8 elasticity/heat element
                           kernels (src/mesh/elements/volume/hexahedron8.cpp,
                           src/assembler/physics/structuralmechanics3d.cpp)
* ``oracle.numbering``  -- node intervals, local DOF numbering and the B1
                           gluing/Dirichlet multiplier numbering
                           (src/mesh/preprocessing/arrangement.cpp,
                           src/assembler/constraints/{constraints,
                           equalityconstraints}.cpp)
* ``oracle.feti``       -- K+ (fix-point regularisation), explicit Schur
                           complements, G/GG^T, projected PCG, lumped and
                           Dirichlet preconditioners, primal recovery
                           (src/solver/specific/itersolver.cpp,
                           src/solver/specific/cpu/itersolvercpu.cpp,
                           src/solver/specific/cluster.cpp)
* ``oracle.htfeti``     -- Hybrid Total FETI: corner nodes, B0 corner gluing,
                           the cluster solve with F0 and S_alpha, cluster
                           kernels (src/mesh/preprocessing/fetidata.cpp,
                           src/solver/specific/cluster.cpp)

Parity pins: the oracle's displacements are checked against the
reference's own regression presets (benchmarks/**/HEXA8*.emr, stored as
fixtures in tests/golden/) and against a global direct solve of the same
assembled system.  The reference itself cannot be built here (MKL, MPI,
METIS), so beyond those presets the 1e-8 parity is pinned to this
restatement.
"""
