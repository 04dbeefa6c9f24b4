"""Synthetic Kuhn-split bump-channel meshes (host-side input generation).

The transonic bump channel used by every benchmark configuration: a box
[0, lx] x [0, ly] x [0, lz] of nx x ny x nz hexahedra, each split into six
tetrahedra by the Kuhn (Freudenthal) construction, interior nodes jittered,
and the lower wall z = 0 lifted by a Gaussian bump blended linearly to zero
at the upper wall.

Construction rules (shared with the reference's synthetic cube generator,
``tests/mesh_utils.py:16-56``, generalised to a non-cubic box):

* node (i, j, k) has index ``i*(ny+1)*(nz+1) + j*(nz+1) + k``, i.e. the
  lexicographic order of ``np.meshgrid(..., indexing="ij")``;
* hexes are visited in the same lexicographic (i, j, k) order, and each hex
  emits six tets, one per axis permutation (a, b, c) in the order
  (0,1,2), (0,2,1), (1,0,2), (1,2,0), (2,0,1), (2,1,0); the tet is the vertex
  walk v0 = (i,j,k), v1 = v0 + e_a, v2 = v1 + e_b, v3 = v2 + e_c, which is
  face-conforming across the whole grid;
* interior nodes (0 < i < nx, 0 < j < ny, 0 < k < nz) move by
  ``rng.uniform(-1, 1, (n_interior, 3)) * jitter * (hx, hy, hz)`` with
  ``rng = np.random.default_rng(seed)``;
* the bump: ``z <- z + h(x) * (1 - z / lz)`` with
  ``h(x) = amplitude * exp(-(x - x_c)**2 / width)``.

Dirichlet boundary: the inflow plane x = 0 and the outflow plane x = lx carry
phi = U * x; all other faces are natural (slip) boundaries.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# Axis-permutation order of the Kuhn split (tests/mesh_utils.py:40).
KUHN_PERMUTATIONS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


@dataclass
class BumpMesh:
    """A generated channel mesh plus its Dirichlet split."""

    nodes: np.ndarray          # (N, 3) float64
    elements: np.ndarray       # (E, 4) int32
    dirichlet_nodes: np.ndarray  # (n_d,) int64, ascending
    shape: tuple               # (nx, ny, nz)
    lengths: tuple             # (lx, ly, lz)

    @property
    def n_nodes(self) -> int:
        return len(self.nodes)

    @property
    def n_tets(self) -> int:
        return len(self.elements)

    def freestream(self, u_inf: float = 1.0) -> np.ndarray:
        return u_inf * self.nodes[:, 0].copy()


def kuhn_box(nx: int, ny: int, nz: int, lx: float = 4.0, ly: float = 1.0,
             lz: float = 1.0):
    """Unjittered Kuhn-split box: (nodes (N,3) f64, elements (E,4) int32)."""
    if min(nx, ny, nz) < 1:
        raise ValueError("kuhn_box needs nx, ny, nz >= 1")
    n_nodes = (nx + 1) * (ny + 1) * (nz + 1)
    if 6 * nx * ny * nz >= 2**31 or n_nodes >= 2**31:
        raise ValueError("mesh too large for int32 connectivity")
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    gx, gy, gz = np.meshgrid(xs, ys, zs, indexing="ij")
    nodes = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)

    stride = np.array([(ny + 1) * (nz + 1), nz + 1, 1], dtype=np.int64)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz),
                             indexing="ij")
    base = (ii.ravel() * stride[0] + jj.ravel() * stride[1] + kk.ravel())
    walk = np.empty((6, 4), dtype=np.int64)
    for p, (a, b, c) in enumerate(KUHN_PERMUTATIONS):
        walk[p, 0] = 0
        walk[p, 1] = stride[a]
        walk[p, 2] = stride[a] + stride[b]
        walk[p, 3] = stride[a] + stride[b] + stride[c]
    elements = (base[:, None, None] + walk[None, :, :]).reshape(-1, 4)
    return nodes, elements.astype(np.int32)


def bump_channel(nx: int, ny: int, nz: int, amplitude: float = 0.05,
                 seed: int = 0, jitter: float = 0.1, lx: float = 4.0,
                 ly: float = 1.0, lz: float = 1.0, bump_center: float = 2.0,
                 bump_width: float = 0.04) -> BumpMesh:
    """The jittered Gaussian-bump channel (see module docstring)."""
    nodes, elements = kuhn_box(nx, ny, nz, lx, ly, lz)
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1),
                             np.arange(nz + 1), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    interior = ((ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)
                & (kk > 0) & (kk < nz))
    rng = np.random.default_rng(seed)
    spacing = np.array([lx / nx, ly / ny, lz / nz])
    if jitter != 0.0:
        shift = rng.uniform(-1.0, 1.0, size=(int(interior.sum()), 3))
        nodes[interior] += shift * (jitter * spacing)
    if amplitude != 0.0:
        x = nodes[:, 0]
        h = amplitude * np.exp(-((x - bump_center) ** 2) / bump_width)
        nodes[:, 2] = nodes[:, 2] + h * (1.0 - nodes[:, 2] / lz)
    dirichlet = np.nonzero((ii == 0) | (ii == nx))[0].astype(np.int64)
    return BumpMesh(nodes=np.ascontiguousarray(nodes),
                    elements=np.ascontiguousarray(elements),
                    dirichlet_nodes=dirichlet, shape=(nx, ny, nz),
                    lengths=(lx, ly, lz))


def smooth_perturbation(nodes: np.ndarray, seed: int, n_modes: int = 4,
                        lengths=(4.0, 1.0, 1.0)) -> np.ndarray:
    """A seeded sum of low-wavenumber sine modes, scaled to max |f| = 1 and
    vanishing on the inflow/outflow planes (so Dirichlet data is unchanged).
    """
    rng = np.random.default_rng(seed)
    lx, ly, lz = lengths
    x, y, z = nodes[:, 0] / lx, nodes[:, 1] / ly, nodes[:, 2] / lz
    f = np.zeros(len(nodes))
    for _ in range(n_modes):
        kx, ky, kz = rng.integers(1, 4, size=3)
        py, pz = rng.uniform(0.0, 2.0 * np.pi, size=2)
        amp = rng.standard_normal()
        f += (amp * np.sin(np.pi * kx * x) * np.cos(np.pi * ky * y + py)
              * np.cos(np.pi * kz * z + pz))
    scale = np.abs(f).max()
    return f / scale if scale > 0 else f


def seeded_state(mesh: BumpMesh, seed: int, u_inf: float = 1.0,
                 amplitude: float = 0.01) -> np.ndarray:
    """phi = U x + amplitude * U * smooth_perturbation (the five seeded
    states of the transonic channel configuration use seeds 0..4)."""
    f = smooth_perturbation(mesh.nodes, seed, lengths=mesh.lengths)
    return u_inf * mesh.nodes[:, 0] + amplitude * u_inf * f


def pocket_state(mesh: BumpMesh, family: str, noise_seed: int = 42,
                 noise: float = 0.005) -> np.ndarray:
    """Supersonic-pocket-bearing potentials: the reference Jacobian test's
    field families (``tests/test_p8_jacobian.py:180-214``) in the unit
    streamwise coordinate s = x / lx, scaled back by lx, plus seeded nodal
    noise that breaks lattice ties."""
    lx = mesh.lengths[0]
    s = mesh.nodes[:, 0] / lx
    if family == "accelerating":
        f = s + 0.3 * s ** 2
    elif family == "shockpoint":
        f = 1.6 * s - 0.3 * s ** 2
    elif family == "mixed":
        f = 1.25 * s + 0.12 * np.sin(2.0 * np.pi * s)
    elif family == "freestream":
        f = s.copy()
    else:
        raise ValueError(f"unknown pocket family {family!r}")
    rng = np.random.default_rng(noise_seed)
    return lx * f + noise * rng.standard_normal(len(s))


def choking_mach(amplitude: float, height: float = 1.0, gamma: float = 1.4) -> float:
    """Freestream Mach at which the bump channel chokes, by the quasi-1-D
    isentropic estimate: the bump spans the channel's width, so its crest
    leaves a throat of (height - amplitude) / height of the inflow area, and
    the mass flux rho q that the Dirichlet inflow and outflow impose cannot
    pass the throat once it exceeds the sonic flux rho* q* (local Mach 1,
    q*^2 = (2 + (gamma - 1) M^2) / ((gamma + 1) M^2) in freestream units).
    Above this Mach the channel has no steady isentropic full-potential
    solution (the supersonic pocket reaches across the throat), so a Newton
    continuation cannot converge there.  Bisection to 1e-12."""
    throat = (height - amplitude) / height
    if not 0.0 < throat <= 1.0:
        raise ValueError("amplitude must lie in [0, height)")

    def sonic_flux(m):
        q2 = (2.0 + (gamma - 1.0) * m * m) / ((gamma + 1.0) * m * m)
        rho = (1.0 + 0.5 * (gamma - 1.0) * m * m * (1.0 - q2)) ** (1.0 / (gamma - 1.0))
        return rho * np.sqrt(q2)

    if throat == 1.0:
        return 1.0
    lo, hi = 1e-3, 1.0
    while hi - lo > 1e-12:
        mid = 0.5 * (lo + hi)
        if sonic_flux(mid) > 1.0 / throat:
            lo = mid
        else:
            hi = mid
    return lo
