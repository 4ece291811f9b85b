"""CPU oracle for the split-step Fourier propagator.

TEST INFRASTRUCTURE ONLY.  Nothing under ``gpe_simulator_b200`` imports this
package; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU baseline leg of
``bench.py`` use it, and only as the checker.

* ``oracle.ssf``   -- NumPy/scipy.fft FP64 restatement of the reference
  propagator (``gpe/make_propagator.py``, ``gpe/make_kernel.py``,
  ``gpe/kernels.py``, ``gpe/helper.py``, ``gpe/nk_extraction.py``).
* ``oracle.expr``  -- evaluator for the reference's potential grammar
  (``config_editor/expressions.py`` / ``gpe/expressions.py``).
* ``oracle.ref_shim`` -- runs the reference's own Python and its CUDA kernel
  strings on the host (only where the reference sources are present); used to
  generate and pin the golden fixtures under ``tests/golden``.
"""
