"""Solver entry point and runtime message channel (mirrors Solver/General)."""
