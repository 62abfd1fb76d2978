"""Checkers for tigre_b200 (test infrastructure only; never imported by the product).

oracle.oracle  -- FP64 host restatement of the reference's projector pair (C++/OpenMP)
oracle.ref     -- the reference's own CUDA build (oracle/_ref), run in child processes
oracle.build   -- build recipe for both
"""
