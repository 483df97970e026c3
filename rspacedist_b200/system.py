"""Host-side set-up of a periodic cell for the real-space hot path: grid,
atom positions, sphere lists and projector tables.

This is the input side of the path (kukan's read_input / pseudocalc set-up);
the arrays it returns are exactly what the device kernels consume:

* grid conventions of read_input_kukan8f.F90:373-385: the cell is
  [-xmax, xmax) per axis with 2*nxmax points, dx = xmax/nxmax, point i at
  (i - 1/2) dx - xmax;
* list vectors of pseudocalc_01b (pseudocalc8f.F90:955-1033) built by the
  library (rs_sphere_lists), with npxmax and num_list chosen as
  tools_listvecdim does (tools8f.F90:240-319);
* projector tables vnlocp(num_list, nprjmx, natom): the dataset's radial
  projector p_{l,i}(r) times the real spherical harmonics of
  pseudocalc8f.F90:2962-2970 times the volume element.  The radial function
  is sampled directly on the coarse grid point instead of going through the
  Fourier filter and double-grid contraction of pseudocalc_07; the tables'
  layout, order (s, p x/y/z per radial, d) and scale match the reference.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass, field

import numpy as np

from . import lib as _lib

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
PSCTOFF = 1.05
NFDG = 4

DIAMOND_BASIS = np.array([
    [0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25],
])


def load_dataset(name: str) -> dict:
    with open(os.path.join(DATA, name + ".json")) as f:
        return json.load(f)


def diamond_positions(ncell: int, a: float, sigma: float = 0.0, seed: int = 0) -> np.ndarray:
    """Diamond-cubic supercell, centred coordinates x = f*A - A/2, Gaussian
    jitter sigma (bohr) from numpy's default_rng(seed)."""
    frac = []
    for i in range(ncell):
        for j in range(ncell):
            for k in range(ncell):
                frac.append((DIAMOND_BASIS + np.array([i, j, k])) / ncell)
    frac = np.concatenate(frac)
    A = ncell * a
    pos = frac * A - A / 2
    if sigma > 0:
        pos = pos + np.random.default_rng(seed).normal(0.0, sigma, pos.shape)
    # keep inside [-A/2, A/2) as the reference's atom shift does
    pos = (pos + A / 2) % A - A / 2
    return pos


def _real_ylm(l: int, x, y, z, r):
    """Real spherical harmonics in the order and normalisation of
    pseudocalc8f.F90:2962-2970 (ylm01..ylm09 times sqfourpi, sq3fourpi...)."""
    pi = np.pi
    with np.errstate(invalid="ignore", divide="ignore"):
        rin = np.where(r > 1e-12, 1.0 / r, 0.0)
    if l == 0:
        return [np.full_like(r, np.sqrt(1.0 / 4.0 / pi))]
    if l == 1:
        c = np.sqrt(3.0 / 4.0 / pi)
        return [c * rin * x, c * rin * y, c * rin * z]
    if l == 2:
        r2 = rin * rin
        return [np.sqrt(15.0 / 16.0 / pi) * r2 * (x * x - y * y),
                np.sqrt(15.0 / 4.0 / pi) * (-r2 * z * x),
                np.sqrt(5.0 / 16.0 / pi) * r2 * (3.0 * z * z - r * r),
                np.sqrt(15.0 / 4.0 / pi) * (-r2 * y * z),
                np.sqrt(15.0 / 4.0 / pi) * r2 * x * y]
    raise ValueError(l)


def projector_layout(ds: dict):
    """[(channel index, l, m)] in the reference's projector order."""
    out = []
    for ci, ch in enumerate(ds["channels"]):
        for m in range(2 * ch["l"] + 1):
            out.append((ci, ch["l"], m))
    # reference order: all of l=0, then l=1 radials, then l=2 (channels are
    # already sorted by (l, i))
    return out


def projector_matrices(ds: dict, key: str) -> np.ndarray:
    """D (key='dion_ha') or S (key='qvd') in projector space."""
    lay = projector_layout(ds)
    P = len(lay)
    m0 = np.array(ds[key])
    M = np.zeros((P, P))
    for a, (ca, la, ma) in enumerate(lay):
        for b, (cb, lb, mb) in enumerate(lay):
            if la == lb and ma == mb:
                sa, sb = ds["channels"][ca]["slot"], ds["channels"][cb]["slot"]
                M[a, b] = 0.5 * (m0[sa][sb] + m0[sb][sa])
    return M


@dataclass
class Cell:
    """One periodic cell with one species (everything the kernels need)."""
    shape: tuple
    h: tuple
    xmax: tuple
    nmax: tuple
    atoms: np.ndarray
    ds: dict
    npmax: tuple = None
    num_list: int = 0
    nprjmx: int = 0
    natinf: np.ndarray = None
    lst: np.ndarray = None
    lstxyz: tuple = None
    natxyz: tuple = None
    vnlocp: np.ndarray = None
    dij: np.ndarray = None
    sss: np.ndarray = None
    extra: dict = field(default_factory=dict)

    @property
    def N(self):
        return int(np.prod(self.shape))

    @property
    def natom(self):
        return len(self.atoms)

    @property
    def dvol(self):
        return self.h[0] * self.h[1] * self.h[2]

    @property
    def nprj(self):
        return np.full(self.natom, self.nprjmx, np.int32)


def make_cell(A, n, atoms, ds, with_s=True, filtered: bool = False, npmesh: int = 2,
              list_builder=None) -> Cell:
    """A: cell edge(s) in bohr, n: grid points per axis (even), atoms (natom,3).
    filtered: the projector tables of pseudocalc_07 (Fourier-filtered radial
    functions on the npmesh double grid, built on the GPU by
    rs_projector_tables) in place of the directly sampled ones.
    list_builder: a function with the arguments and results of
    rs_sphere_lists (see sphere_lists_library) that builds the list vectors;
    None uses the library's."""
    A = np.broadcast_to(np.asarray(A, float), (3,))
    n = np.broadcast_to(np.asarray(n, int), (3,))
    if np.any(n % 2):
        raise ValueError("grid sizes must be even (2*nxmax)")
    nmax = tuple(int(v) // 2 for v in n)
    xmax = tuple(float(a) / 2 for a in A)
    h = tuple(xmax[i] / nmax[i] for i in range(3))
    cell = Cell(shape=tuple(int(v) for v in n), h=h, xmax=xmax, nmax=nmax,
                atoms=np.asarray(atoms, float).reshape(-1, 3), ds=ds)
    build_lists(cell, list_builder)
    build_projectors(cell, with_s=with_s)
    if filtered:
        from .projectors import projector_tables
        cell.vnlocp = projector_tables(cell, npmesh=npmesh)
    return cell


def list_dims(cell: Cell):
    """npxmax and num_list as tools_listvecdim chooses them (auto mode)."""
    rc = cell.ds["rcut"] * PSCTOFF
    npm, nl = [], []
    for ax in range(3):
        npx = max(1, int(rc / cell.h[ax]) + 1 + NFDG)
        ncp = cell.shape[ax]
        if 2 * cell.nmax[ax] < 2 * npx:
            nlx = 2 * npx
        elif ncp > 2 * npx:
            nlx = 2 * npx
        else:
            nlx = ncp
        npm.append(npx)
        nl.append(nlx)
    return tuple(npm), int(np.prod(nl))


def sphere_lists_library(atoms, rcut, nmax, h, npmax, nfdg, num_list):
    """List vectors of pseudocalc_01b by the library (rs_sphere_lists):
    returns natx, naty, natz, natinf, lst, lstx, lsty, lstz."""
    A = len(atoms)
    at = np.ascontiguousarray(atoms, dtype=np.float64)
    ax, ay, az = (np.ascontiguousarray(at[:, k]) for k in range(3))
    rc = np.full(A, rcut)
    nat = [np.zeros(A, np.int32) for _ in range(3)]
    natinf = np.zeros(A, np.int32)
    lst = np.zeros(A * num_list, np.int32)
    lx, ly, lz = (np.zeros(A * num_list, np.int32) for _ in range(3))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    _lib.call("rs_sphere_lists", A, dp(ax), dp(ay), dp(az), dp(rc), nmax[0], nmax[1], nmax[2],
              h[0], h[1], h[2], npmax[0], npmax[1], npmax[2], nfdg, num_list, ip(nat[0]),
              ip(nat[1]), ip(nat[2]), ip(natinf), ip(lst), ip(lx), ip(ly), ip(lz))
    return nat[0], nat[1], nat[2], natinf, lst, lx, ly, lz


def build_lists(cell: Cell, list_builder=None):
    npmax, num_list = list_dims(cell)
    fn = list_builder or sphere_lists_library
    nx_, ny_, nz_, natinf, lst, lx, ly, lz = fn(cell.atoms, cell.ds["rcut"] * PSCTOFF, cell.nmax,
                                                 cell.h, npmax, NFDG, num_list)
    cell.npmax, cell.num_list = npmax, num_list
    cell.natinf, cell.lst = natinf, lst
    cell.lstxyz = (lx, ly, lz)
    cell.natxyz = (nx_, ny_, nz_)


def build_projectors(cell: Cell, with_s=True):
    ds = cell.ds
    lay = projector_layout(ds)
    P = len(lay)
    A, L = cell.natom, cell.num_list
    dx, dy, dz = cell.h
    v = np.zeros((A, P, L))
    dr = ds["dr"]
    chans = [np.asarray(c["p"]) for c in ds["channels"]]
    rcut = ds["rcut"]
    lx, ly, lz = (a.reshape(A, L) for a in cell.lstxyz)
    for a in range(A):
        n = int(cell.natinf[a])
        tx = cell.atoms[a, 0] - (cell.natxyz[0][a] * dx - 0.5 * dx)
        ty = cell.atoms[a, 1] - (cell.natxyz[1][a] * dy - 0.5 * dy)
        tz = cell.atoms[a, 2] - (cell.natxyz[2][a] * dz - 0.5 * dz)
        x = lx[a, :n] * dx - tx
        y = ly[a, :n] * dy - ty
        z = lz[a, :n] * dz - tz
        r = np.sqrt(x * x + y * y + z * z)
        inside = r < rcut
        ylm = {l: _real_ylm(l, x, y, z, r) for l in (0, 1, 2)}
        for j, (ci, l, m) in enumerate(lay):
            pr = np.interp(r, np.arange(len(chans[ci])) * dr, chans[ci])
            v[a, j, :n] = np.where(inside, pr * ylm[l][m] * cell.dvol, 0.0)
    cell.nprjmx = P
    cell.vnlocp = v
    D = projector_matrices(ds, "dion_ha")
    cell.dij = np.ascontiguousarray(np.broadcast_to(D, (A, P, P)))
    if with_s and ds["kind"] == "paw":
        S = projector_matrices(ds, "qvd")
        cell.sss = np.ascontiguousarray(np.broadcast_to(S, (A, P, P)))
    else:
        cell.sss = None


def smooth_veff(cell: Cell, seed: int = 0, amp: float = 0.3) -> np.ndarray:
    """A smooth periodic synthetic local potential (a few low Fourier modes)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = cell.shape
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx,
                          indexing="ij")
    v = np.zeros((nz, ny, nx))
    for _ in range(6):
        k = rng.integers(-2, 3, 3)
        ph = rng.uniform(0, 2 * np.pi)
        v += amp * rng.uniform(-1, 1) * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + ph)
    return v.ravel() - 0.5


def random_bands(cell: Cell, nb: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nb, cell.N)) * 0.1


def small_cell_set(count: int = 32, seed: int = 2, spacing: float = 0.30):
    """Independent small periodic cells, alternately Si8 (PAW dataset) and C8
    (NC dataset) diamond cubic: lattice constants 10.26 / 6.74 bohr scaled by
    U[0.97, 1.03], atoms jittered by 0.03 bohr, grids of even size with
    spacing close to `spacing` (about 22^3 to 36^3)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        name, a0 = (("si_paw", 10.26), ("c_ncps", 6.74))[k % 2]
        a = a0 * rng.uniform(0.97, 1.03)
        n = 2 * int(round(a / (2 * spacing)))
        pos = diamond_positions(1, a, 0.03, int(rng.integers(1 << 30)))
        out.append(make_cell(a, n, pos, load_dataset(name)))
    return out
