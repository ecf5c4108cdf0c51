"""Names of the golden cases (tests/golden/make_golden.py) the CPU tests check."""
CASES_FOR_TESTS = ("cube3d", "film2d")
