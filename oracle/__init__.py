"""Parity oracles for the orientation search -- test infrastructure only."""
