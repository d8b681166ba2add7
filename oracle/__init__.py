"""ORACLE package — test infrastructure only (see oracle.py)."""
