"""B200-native DFT-D3 dispersion correction.

Python interface of the CUDA library in ``../lib``, mirroring the reference's
``dftd3`` package (``dftd3.interface``, ``dftd3.library``): the same classes,
argument names and error behaviour, with a GPU-evaluated hot path.
"""

__version__ = "1.6.0"
