"""ORACLE / TEST INFRASTRUCTURE ONLY.

CPU restatement of redbirdpy's FEM forward / Jacobian / Gauss-Newton path,
used as the checker for the CUDA implementation in ``redbirdpy_b200`` and as
the timed CPU baseline of ``bench.py``.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline leg and its
``--impl reference`` arm) may import it; the product package never does.

Parity pinning: every function here is checked against golden fixtures that
were produced by running the reference redbirdpy 0.2.0 itself in this
container (``tests/golden/make_golden.py``), see ``tests/test_oracle.py``.
"""

from . import femoracle, tsearch  # noqa: F401
