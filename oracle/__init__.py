"""Test-only checkers: the CPU restatement of the reference kernels and a
launcher for the reference's own kernels.  Nothing in the product imports
this package."""
