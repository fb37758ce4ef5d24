"""CPU oracle for the GraphGP hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy (plus a small C file for the k-NN traversal at large sizes), the reference
algorithms of stanford-ism/graphgp for the path this repository accelerates:

* ``tree.py``   -- k-d tree build and preceding-k-NN query  (reference ``graphgp/tree.py``)
* ``graph.py``  -- depths, ordering by depth, offsets, ``check_graph`` (reference ``graphgp/graph.py``)
* ``refine.py`` -- covariance lookup, dense root, refine / inverse / logdet, generate (reference
  ``graphgp/refine.py``)
* ``extras.py`` -- kernel tables (reference ``graphgp/extras.py``)
* ``adjoint.py`` -- reverse-mode gradient of generate / logdet (what JAX autodiff computes through
  reference ``graphgp/refine.py:123-145``), written out by hand
* ``jax_random.py`` -- JAX's threefry PRNG, to regenerate the reference tests' random inputs

Parity is pinned against the reference's own tests: the portable known answers
(``tests/test_tree.py:19-24``, ``tests/test_graph.py:40-82``) and the RNG-bound goldens
(``tests/test_tree.py:27-32``, ``tests/test_graph.py:14-27``, ``tests/test_refine.py:29-43``), whose inputs
``jax_random`` reproduces bit-for-bit (sentinel ``points[0,0] == -0.61777326``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import this package,
and only as the checker or the timed CPU baseline. The product (``graphgp_b200``) never imports it and
has no CPU fallback.
"""
