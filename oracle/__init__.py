"""CPU oracle of the SpGEMM hot path — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
legs, as the checker and the timed CPU baseline; the engine never uses it.
"""
from .oracle import (checksum, gen_stencil27, max_threads, multiply, multiply_rows, products,  # noqa: F401
                     rows_stream, transpose)
