"""Empty matplotlib stand-in so the reference lcode package imports; no
plotting is reached by the fixture generator."""
