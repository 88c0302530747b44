"""CPU oracle (test infrastructure only): a restatement of the reference
lcodePy 3D algorithm used to check the CUDA product.  Never imported by the
product package."""
