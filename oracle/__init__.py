"""Test infrastructure: the CPU oracle of the SIMPLEC path (never imported by the product)."""
