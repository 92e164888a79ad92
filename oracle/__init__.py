"""ORACLE -- test infrastructure only (the checker, never the product).

Two CPU implementations of oneDAL's dense k-means Lloyd path:

* ``oracle.restated``: a plain-C restatement (oracle/kmeans_oracle.c) of the
  DAAL kernel's semantics, built by ``oracle.build``;
* ``oracle.daal_ref``: the reference's own DAAL kernel compiled from its sources
  (oracle/ref/Makefile -> oracle/_ref/libkmeans_daal_ref.so).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this package.
"""
