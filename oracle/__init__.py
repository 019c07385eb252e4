"""Parity oracles for the FDK engine (test infrastructure only)."""
