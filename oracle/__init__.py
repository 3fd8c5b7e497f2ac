"""CPU FP64 oracle of the FLURSYS projection path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
as the checker (never as the thing measured for the GPU arm).
"""
