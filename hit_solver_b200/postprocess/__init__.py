"""Post-processing of HIT runs on the device (the reference's
``OOP/postprocess`` package): shell spectra."""

from .spectra import HIT2DSpectra, SpectrumResults2D, shell_spectra, state_shell_spectra

__all__ = ["HIT2DSpectra", "SpectrumResults2D", "shell_spectra", "state_shell_spectra"]
