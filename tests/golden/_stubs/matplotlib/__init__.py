"""Placeholder so the reference's modules import without matplotlib (plotting is
not exercised when golden vectors are generated)."""
