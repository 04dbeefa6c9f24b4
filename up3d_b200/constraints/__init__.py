"""Constraints of the lifting solves on the device (pyfp3d/constraints)."""
