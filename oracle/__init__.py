"""Test infrastructure: CPU restatement of the reference hot path (the checker).

Nothing on the product path imports this package.
"""
