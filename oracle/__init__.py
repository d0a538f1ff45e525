"""ORACLE -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It holds:

* ``v2rdm_oracle.c``  -- a plain-C restatement of hilbert's v2RDM constraint
  maps, index tables, b, c and guess (C1 symmetry), loaded through ctypes
  (``oracle.maps``);
* ``bpsdp.py``        -- a numpy restatement of the boundary-point SDP
  iteration (Povh, Rendl & Wiegele 2006; Malick et al. 2009) with the outer
  protocol hilbert drives (``oracle.bpsdp``);
* ``build_ref.sh``    -- the recipe that compiles hilbert's own map sources
  into ``oracle/_ref/libv2rdm_ref.so`` (``oracle.ref``), the bit-exact pin
  for the restatement.
"""
