"""CPU oracles for the lex+parse path. TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may use this package, and only as the checker or the baseline.

* ``ref``    - the reference's own C backend (oracle/_ref, built by build_ref.py).
* ``port``   - a C restatement of that backend (oracle/oracle.c) taking the
               grammar tables at run time.
"""
