"""CPU FP64 oracle for the UPPE right-hand side and the RK45 integrator.

TEST INFRASTRUCTURE ONLY. This package restates, in numpy, the reference algorithm
(Luna.jl v0.6.2) of the hot path so that the CUDA implementation can be checked
against it. Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it. The product (``luna.jl_b200``)
never does: its right-hand side and integrator run on the GPU only.

Parity pin: the restatement is checked against the reference's own known answers
(``test/test_gnlse.jl:51,55`` soliton self-frequency shift, ``test/test_rk45.jl``
soliton recovery, ``test/test_kerr.jl``, ``test/test_ionisation.jl``,
``test/test_raman.jl``), because the Julia reference cannot run in this environment.
"""
