"""Linear and nonlinear solvers on the device (pyfp3d.solve)."""
