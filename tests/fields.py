"""Initial conditions shared by the tests: the package's seeded generators."""
from spooky_b200.initial import grid, kvectors, random_solenoidal, to_spectral  # noqa: F401
