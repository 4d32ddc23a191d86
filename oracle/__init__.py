"""CPU oracle for the Fourier-slice + CTF image-simulation path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``cryojax_b200`` package imports
this directory: it is the checker, used by ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py``.  It is a float64 NumPy restatement of cryoJAX's
``FourierSliceExtraction`` / ``AstigmaticCTF`` / ``LinearImageModel`` path;
each function cites the cryoJAX file and line it follows.
"""
