"""CPU parity oracle for the fast_shepherd_score_b200 hot path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this package,
and only as the checker or the timed CPU baseline -- never as the thing measured or
shipped.  The product package never imports it and has no CPU fallback.

What it restates (reference = shepherd_score, file paths relative to its repo root):

* ``libfss_oracle.so`` (``fss_oracle.c``): the numba value+gradient kernels of
  ``shepherd_score/accel/kernels/cpu.py`` and the fused CPU fine loop of
  ``shepherd_score/accel/kernels/cpu_fused.py`` (fp64 accumulation, fp32 state).
* :mod:`oracle.seeds`: ``batched_seeds_torch`` (``shepherd_score/accel/drivers/_common.py:281``)
  in numpy, including the fp64 closed-form PCA.
* :mod:`oracle.align`: the batched drivers ``coarse_fine_align_many``
  (``accel/drivers/shape.py:155``), ``coarse_fine_esp_align_many`` (``accel/drivers/esp.py:139``),
  ``coarse_fine_pharm_align_many`` (``accel/drivers/pharm.py:123``) and the shape+pharm combined
  loop composed from ``cpu_fused._tail_vol_color`` (``cpu_fused.py:112``).
* :mod:`oracle.scores`: fp64 numpy scoring (``score/gaussian_overlap.py:16``,
  ``score/electrostatic_scoring.py:17``, ``score/pharmacophore_scoring.py``) for the score and
  coordinate-gradient checks.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference itself (imported from
its source tree, numba path) on seeded inputs and commits the outputs under ``tests/golden``;
``tests/test_oracle_golden.py`` checks this oracle against them.
"""
