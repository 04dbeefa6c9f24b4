"""Wall post-processing on the device (pyfp3d/post)."""
