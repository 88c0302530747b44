"""B200-native quasistatic 3D xi-step engine with lcodePy's Simulation API."""
__version__ = "0.1.0"
