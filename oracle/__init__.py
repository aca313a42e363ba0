"""Parity checker for the MD path (test infrastructure only; see oracle.py)."""
