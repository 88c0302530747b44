"""Empty pyplot stand-in (see package docstring)."""
