"""ORACLE — test infrastructure only (see refcpu.cpp's header).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference arms; never by the product package.
"""
