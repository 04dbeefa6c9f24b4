"""up3d_b200 -- B200-native (sm_100a) element-loop hot path of the pyfp3d
full-potential solver.

Drop-in modules mirror the reference package layout:

    up3d_b200.kernels.jacobian   PicardOperator
    up3d_b200.kernels.upwind     UpwindOperator
    up3d_b200.kernels.gradient   element_velocity_q2
    up3d_b200.physics.isentropic isentropic scalars and device field sweeps
    up3d_b200.solve.linear       SpMV-based CG / GMRES and preconditioners
    up3d_b200.solve.fused        fused residual + Jacobian evaluation

All device work goes through the C ABI in include/up3d.h
(up3d_b200/lib/libup3d.so); there is no CPU fallback.
"""

__version__ = "0.1.0"
