"""Isentropic physics (pyfp3d.physics)."""
