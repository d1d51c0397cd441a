"""Empty stand-in for sigpy.mri (only the out-of-scope CLI scripts use it)."""
