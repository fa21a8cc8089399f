"""CPU FP64 oracle of the HEXA(T) inner solve path -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this
package, as the checker or as the timed CPU baseline; the product never does.
Parity is unpinned: the reference ships no golden vectors (see
hexat_oracle.c).
"""
