"""Placeholder pyplot: any attribute access raises, plotting is never called."""


def __getattr__(name):
    raise RuntimeError(f"matplotlib.pyplot.{name} is not available in golden-vector generation")
