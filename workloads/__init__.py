"""Benchmark and test workloads: the reference's test systems, the benchmark
configurations' seeded inputs and the ahead-of-time build of their kernels.

Input generation only -- not part of the solver package.
"""
