"""MEX runtime stand-in (test infrastructure): see matrix.h."""
