"""CPU ORACLE for the gpusketch_b200 tests.  TEST INFRASTRUCTURE ONLY.

Two checkers, both built by ``make -f oracle/Makefile`` (called from __graft_entry__.build()):

* ``Restatement`` binds oracle/_build/libgsoracle.so, a plain-C restatement of the reference's
  sketch update / sample / Boruvka / k-forest arithmetic (oracle/gsoracle.c cites the reference
  file:line of every function).
* ``RefCC`` / ``RefMC`` bind oracle/_ref/libgsref.so, the reference's own CCSketchAlg and
  MCSketchAlg compiled from its sources (oracle/refshim/*.cpp wrap them in extern "C").

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this package; the
product (gpusketch_b200) never imports it.
"""
from .bridge import RefCC, RefMC, Restatement, bucket_by_vertex, ref_available

__all__ = ["RefCC", "RefMC", "Restatement", "bucket_by_vertex", "ref_available"]
