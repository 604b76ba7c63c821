"""CPU oracle for the density-fitting J/K path — TEST INFRASTRUCTURE ONLY.

This package is a numpy restatement of dftax's density-fitting path, used as
the checker of the CUDA library. Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / reference arm may import it; the product
(``dftax_b200``) never does and has no CPU fallback.

Parity is pinned: ``tests/golden/*.npz`` are outputs of the reference's own
functions (run by ``tests/golden/make_golden.py``), and
``tests/test_oracle_golden.py`` checks this oracle against them (Boys table and
values, basis normalization and cart2sph, the bucketed 3-center and 2-center
integrals, the metric pseudo-inverse, the DF energy, J and K).

Modules:
  boys   — ``dftax/energy/boys.py`` (table scheme, Taylor, asymptotic, exact)
  md     — ``dftax/integrals/eri3c_bucketed.py`` (shells, plan, E/R tables,
           per-class 3-center and 2-center integrals, block cart->sph) and the
           Schwarz shell-pair keep (``eri3c_bucketed.py:140-169``)
  df     — ``dftax/ks/terms.py`` (metric pseudo-inverse, DFCoulomb energy,
           RI-K factor and orbital recovery) and ``dftax/energy/hybrid.py``
           (DF-K), with J and K as the analytic gradients of the energy.
  cpu    — the same 3-center and 2-center integrals compiled (``cpu_df.cpp``,
           C++ on all host threads) and a full DF build with dftax's J/K
           contractions: the timed CPU baseline of ``bench.py``, checked
           against the golden fixtures and against ``md``
           (``tests/test_oracle_cpu.py``).
"""
