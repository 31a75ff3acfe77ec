"""Test infrastructure: CPU restatement of the reference render path and the reference build recipe.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs use this package,
as the checker. The product path never imports it.
"""
