"""CPU oracle for the dedispersion path -- TEST INFRASTRUCTURE ONLY.

Used by ``tests/``, ``__graft_entry__.smoke()`` (as the checker) and the
CPU-baseline leg of ``bench.py``.  The product package never imports it.
"""
