"""Experimental solvers (reference: chromatix/experimental)."""
