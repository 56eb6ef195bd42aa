"""NumPy/SciPy-backed stand-in for ``cupyx`` (fixture generation only)."""
