"""Single-rank stand-in for mpi4py, used only to import the reference lcode
package in the fixture generator (tests/golden/make_golden.py)."""
