"""Drop-in element kernels (pyfp3d.kernels)."""
