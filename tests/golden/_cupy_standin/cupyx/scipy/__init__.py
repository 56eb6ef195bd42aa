"""NumPy/SciPy-backed stand-in for ``cupyx.scipy`` (fixture generation only)."""
