"""ORACLE -- test infrastructure, not product code.

CPU restatements of the reference's algorithms for the hot paths, each
function citing the reference file:line it follows.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` import this package, and only as the checker.  The product
package (``cat_surface_gpu_b200``) never imports it and has no CPU fallback.
"""
