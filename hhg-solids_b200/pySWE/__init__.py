"""ctypes API of the hhg-b200 SBE propagator, with the classes of the reference's pySWE."""
from .pyswe import SWE, SWEBatch, SWEServer, Settings, SWEError, default_library, harmonic_intensities, spectrum  # noqa: F401
