"""Empty stand-in for sigpy.plot."""
