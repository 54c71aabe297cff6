"""Synthetic diamond cells with analytic local potential and KB-type projectors.

Builds, in FP64 on the host, exactly the inputs the reference's Hamiltonian
consumes, so that the CPU oracle, the reference harness and the GPU engine all
see bit-identical arrays:

* grid: nx*ny*nz periodic points, spacing h = a/N per axis, points at h*i
  (GridRange {0,0,0,N}, the reference's convention);
* V(r) = sum_atoms -4 exp(-d^2 / (2*0.7^2)) Ha with d the minimum-image
  distance, folded per axis like ``fold`` (PseudoPotOperator.h:14);
* projectors per atom: k=0 (l=0, E=+2 Ha) and k=1 (l=1, E=-1 Ha), radial
  w_l(r) = r^l exp(-r^2/(2*0.6^2)) for r <= 2.5 bohr, else 0, tabulated on the
  cube ``GridForSphere`` returns (GridSubgrid.h:482-492) around the unwrapped
  atom position, the way mMakeSubspacePPnonlocal_Radial fills it
  (PseudoPotOperator.h:473-565);
* Y_lm on the same cube as ``SetYlmAround`` (PseudoPotOperator.h:27-71):
  Y00 = 1/sqrt(4 pi); Y1,-1 / Y1,0 / Y1,1 = sqrt(3/(4 pi)) * (y, z, x)/r,
  and the value at r^2 < 1e-14 is Y00 for l = 0 and 0 otherwise.

The flat arrays returned by :meth:`Cell.desc_arrays` are the reference's
per-atom cube tables (PP_nonlocal_each_atom, PseudoPotOperator.h:21-24).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# fractional sites of the 8-atom cubic diamond cell (input/diamond8.txt:23-30)
DIAMOND_SITES = np.array(
    [
        [0.00, 0.00, 0.00],
        [0.25, 0.25, 0.25],
        [0.50, 0.50, 0.00],
        [0.75, 0.75, 0.25],
        [0.50, 0.00, 0.50],
        [0.75, 0.25, 0.75],
        [0.00, 0.50, 0.50],
        [0.25, 0.75, 0.75],
    ],
    dtype=np.float64,
)
A0 = 6.74          # bohr, 8-atom cell edge
N0 = 40            # grid points per 8-atom cell edge
V_DEPTH = -4.0
V_SIGMA = 0.7
PROJ_SIGMA = 0.6
PROJ_CUTOFF = 2.5
PROJ_L = (0, 1)
PROJ_E = (2.0, -1.0)
Y00 = 1.0 / math.sqrt(4.0 * math.pi)
Y1C = math.sqrt(3.0 / (4.0 * math.pi))


def grid_for_sphere(R, rc, h):
    """GridForSphere (GridSubgrid.h:482-492): [begin, end) per axis."""
    begin = [int(math.ceil((R[i] - rc) / h[i] - 0.5)) for i in range(3)]
    end = [int(math.floor((R[i] + rc) / h[i] + 0.5)) + 1 for i in range(3)]
    return begin, end


def _fold(x, box):
    """fold (PseudoPotOperator.h:14): minimum image per axis."""
    return np.where(x * 2.0 > box, x - box, np.where(x * 2.0 < -box, x + box, x))


@dataclass
class Cell:
    nx: int
    ny: int
    nz: int
    hx: float
    hy: float
    hz: float
    positions: np.ndarray                 # (na, 3) bohr
    V: np.ndarray = field(repr=False)     # (N,) FP64
    proj_l: tuple = PROJ_L
    proj_E: tuple = PROJ_E
    cutoff: float = PROJ_CUTOFF
    fd_order: int = 8
    # per atom, per projector: (begin[3], size[3], w cube); per atom, per lm: Y cube
    cubes: list = field(default_factory=list, repr=False)
    w_tabs: list = field(default_factory=list, repr=False)
    ylm_tabs: list = field(default_factory=list, repr=False)

    @property
    def N(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def dV(self) -> float:
        return self.hx * self.hy * self.hz

    @property
    def n_atoms(self) -> int:
        return int(self.positions.shape[0])

    @property
    def n_lm(self) -> int:
        return (max(self.proj_l) + 1) ** 2 if self.proj_l else 0

    def desc_arrays(self):
        """Flat arrays in the reference's cube-table form (see module doc)."""
        na, npj, nlm = self.n_atoms, len(self.proj_l), self.n_lm
        cube = np.zeros((na, npj, 6), dtype=np.int32)
        w_off = np.zeros(na * npj, dtype=np.int64)
        ylm_off = np.zeros(na * nlm, dtype=np.int64)
        w_parts, y_parts = [], []
        off = 0
        for a in range(na):
            for k in range(npj):
                b, s, w = self.cubes[a][k]
                cube[a, k, :3] = b
                cube[a, k, 3:] = s
                w_off[a * npj + k] = off
                w_parts.append(w)
                off += w.size
        w_data = np.concatenate(w_parts) if w_parts else np.zeros(1)
        off = 0
        for a in range(na):
            for lm in range(nlm):
                y = self.ylm_tabs[a][lm]
                ylm_off[a * nlm + lm] = off
                y_parts.append(y)
                off += y.size
        ylm_data = np.concatenate(y_parts) if y_parts else np.zeros(1)
        return dict(
            cube=np.ascontiguousarray(cube.reshape(-1)),
            w_data=np.ascontiguousarray(w_data, dtype=np.float64),
            w_off=w_off,
            ylm_data=np.ascontiguousarray(ylm_data, dtype=np.float64),
            ylm_off=ylm_off,
            proj_l=np.array(self.proj_l, dtype=np.int32),
            proj_E=np.array(self.proj_E, dtype=np.float64),
            atom_pos=np.ascontiguousarray(self.positions.reshape(-1), dtype=np.float64),
            V=np.ascontiguousarray(self.V, dtype=np.float64),
        )


def _ylm_cube(l, m, begin, size, R, h):
    ix = np.arange(size[0]) + begin[0]
    iy = np.arange(size[1]) + begin[1]
    iz = np.arange(size[2]) + begin[2]
    z = (h[2] * iz - R[2])[:, None, None]
    y = (h[1] * iy - R[1])[None, :, None]
    x = (h[0] * ix - R[0])[None, None, :]
    rr = x * x + y * y + z * z
    small = rr < 1.0e-14
    r = np.sqrt(np.where(small, 1.0, rr))
    if l == 0:
        val = np.full(rr.shape, Y00)
    elif l == 1:
        comp = {-1: y, 0: z, 1: x}[m]
        val = Y1C * (np.broadcast_to(comp, rr.shape) / r)
        val = np.where(small, 0.0, val)
    else:
        raise NotImplementedError("analytic Y_lm tables are built for l <= 1")
    return np.ascontiguousarray(val.reshape(-1), dtype=np.float64)


def _w_cube(l, begin, size, R, h, rc, sigma):
    ix = np.arange(size[0]) + begin[0]
    iy = np.arange(size[1]) + begin[1]
    iz = np.arange(size[2]) + begin[2]
    rz2 = ((h[2] * iz - R[2]) ** 2)[:, None, None]
    ry2 = ((h[1] * iy - R[1]) ** 2)[None, :, None]
    rx2 = ((h[0] * ix - R[0]) ** 2)[None, None, :]
    rr = rx2 + ry2 + rz2
    g = np.exp(-rr / (2.0 * sigma * sigma))
    if l == 0:
        val = g
    else:
        val = np.sqrt(rr) ** l * g
    val = np.where(rr > rc * rc, 0.0, val)
    return np.ascontiguousarray(val.reshape(-1), dtype=np.float64)


def build_cell(reps=(1, 1, 1), n_per_cell=N0, a0=A0, displacement=0.0, seed=0,
               fd_order=8, grid=None, nonlocal_on=True, potential_on=True):
    """Diamond supercell reps[0] x reps[1] x reps[2] of the 8-atom cell.

    ``grid`` overrides the point counts (nx, ny, nz) (used for small test
    cells); by default each 8-atom cell edge carries ``n_per_cell`` points.
    ``displacement`` is the standard deviation (bohr) of seeded Gaussian
    displacements of every atom.
    """
    rx, ry, rz = reps
    Lx, Ly, Lz = a0 * rx, a0 * ry, a0 * rz
    if grid is None:
        nx, ny, nz = n_per_cell * rx, n_per_cell * ry, n_per_cell * rz
    else:
        nx, ny, nz = grid
    hx, hy, hz = Lx / nx, Ly / ny, Lz / nz
    pos = []
    for k in range(rz):
        for j in range(ry):
            for i in range(rx):
                for f in DIAMOND_SITES:
                    pos.append([(f[0] + i) * a0, (f[1] + j) * a0, (f[2] + k) * a0])
    pos = np.array(pos, dtype=np.float64)
    if displacement > 0.0:
        rng = np.random.default_rng(seed)
        pos = pos + rng.normal(0.0, displacement, size=pos.shape)

    # local potential, minimum image per axis
    V = np.zeros((nz, ny, nx), dtype=np.float64)
    if potential_on:
        xs = hx * np.arange(nx)
        ys = hy * np.arange(ny)
        zs = hz * np.arange(nz)
        inv = 1.0 / (2.0 * V_SIGMA * V_SIGMA)
        for R in pos:
            dx2 = _fold(xs - R[0], Lx) ** 2
            dy2 = _fold(ys - R[1], Ly) ** 2
            dz2 = _fold(zs - R[2], Lz) ** 2
            rr = dz2[:, None, None] + dy2[None, :, None] + dx2[None, None, :]
            V += V_DEPTH * np.exp(-rr * inv)
    cell = Cell(nx, ny, nz, hx, hy, hz, pos, V.reshape(-1), fd_order=fd_order)
    if not nonlocal_on:
        cell.proj_l, cell.proj_E = (), ()
        cell.positions = pos
        cell.cubes = [[] for _ in range(len(pos))]
        cell.ylm_tabs = [[] for _ in range(len(pos))]
        return cell
    h = (hx, hy, hz)
    nlm = cell.n_lm
    for R in pos:
        per_k = []
        for l in cell.proj_l:
            b, e = grid_for_sphere(R, cell.cutoff, h)
            size = [e[i] - b[i] for i in range(3)]
            per_k.append((b, size, _w_cube(l, b, size, R, h, cell.cutoff, PROJ_SIGMA)))
        cell.cubes.append(per_k)
        ys = []
        for lm in range(nlm):
            l = int(math.isqrt(lm))
            m = lm - l * l - l
            kf = cell.proj_l.index(l)
            b, size, _ = per_k[kf]
            ys.append(_ylm_cube(l, m, b, size, R, h))
        cell.ylm_tabs.append(ys)
    return cell


def initial_states(ns, N, seed=1234, dtype=np.float64):
    """Seeded uniform(-0.5, 0.5) states, state-major (ns, N)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-0.5, 0.5, size=(ns, N)).astype(dtype)


# The configurations the engine is measured on (sizes per the 8-atom cell edge).
CONFIGS = {
    "diamond8_40": dict(reps=(1, 1, 1)),                           # 8 atoms, 40^3, 16 states
    "diamond64_80": dict(reps=(2, 2, 2)),                          # 64 atoms, 80^3, 256 states
    "diamond216_120": dict(reps=(3, 3, 3), displacement=0.05),     # 216 atoms, 120^3, 480 states
}
