"""kukan's restart files, so that GPU runs restart from and hand off to kukan.

The files are Fortran unformatted sequential files as gfortran writes them:
each record is a 4-byte little-endian length, the data, and the length again.
A record longer than 2**31 - 9 bytes is split into subrecords: a leading
marker is negative when another subrecord follows, a trailing marker when
another one precedes.  The record sequences follow rw_wfpot8f.F90:

* ``wfc.NNNNN.MMM`` (write_wf, rw_wfpot8f.F90:352-395; read_wf :7-190):
  version 5; (nrc, nums, ncol, neigmx, numk, ncpx, ncpy, ncpz);
  (nrx, nry, nrz, myr_kpt); ksym; sval(neigmx, nums+1-ncol, numk); then one
  record per band, spin and k point holding svecre(:,:,:,l,ns,nk) (real*8,
  x fastest).
* ``rho.NNNNN`` / ``r_o.NNNNN`` (write_rhovht :398-470; read_rho :193-306):
  version 3; (nspv, ncpx, ncpy, ncpz, nradmx, npoint, num_atcell);
  (nrx, nry, nrz); (na_atcell, natcell_inf(num_atcell)); rhosmt;
  rhotrur(:,:,:,1:num_atcell); rhosmtr(:,:,:,1:num_atcell).
* ``vht.NNNNN`` (write_rhovht :472-483; read_vht :309-348): version 3;
  (ncpx, ncpy, ncpz, nmesh); (nrx, nry, nrz); vh_dense.

File names come from get_fname (:535-572): the name, then the rank as five
zero-padded digits and, for wave functions, the k-point rank as three.

Bands move between the device and the file one record at a time, so a
1100-band Si512 set (9 GB as FP32) never needs a second full copy in host
memory.  FP32 bands are widened to real*8 on write and rounded on read.
"""
from __future__ import annotations

import os
import struct
from typing import BinaryIO, Iterable, Sequence

import numpy as np

WFC_VERSION = 5
RHO_VERSION = 3
VHT_VERSION = 3
_MAX_SUB = 2 ** 31 - 9  # largest gfortran subrecord


def fname(name: str, nr1: int, nr2: int = -1) -> str:
    """get_fname: 'wfc.00000.000' style names (nr2 < 0: 'rho.00000')."""
    if nr1 >= 10 ** 5 or nr2 >= 10 ** 3:
        raise ValueError("get_fname: not enough digits")
    return f"{name}.{nr1:05d}" + (f".{nr2:03d}" if nr2 >= 0 else "")


# ------------------------------------------------------------------ records
def write_record(f: BinaryIO, *parts) -> None:
    """One Fortran record holding the concatenated bytes of `parts` (numpy
    arrays in Fortran order, or bytes)."""
    data = b"".join(p if isinstance(p, (bytes, bytearray)) else
                    np.asarray(p).tobytes(order="F") for p in parts)
    n = len(data)
    if n <= _MAX_SUB:
        f.write(struct.pack("<i", n))
        f.write(data)
        f.write(struct.pack("<i", n))
        return
    pos = 0
    while pos < n:
        m = min(_MAX_SUB, n - pos)
        last = pos + m >= n
        f.write(struct.pack("<i", m if last else -m))  # negative: more follow
        f.write(data[pos:pos + m])
        f.write(struct.pack("<i", -m if pos > 0 else m))  # negative: some precede
        pos += m


def read_record(f: BinaryIO) -> bytes:
    """The bytes of the next record (subrecords joined)."""
    out = []
    while True:
        head = f.read(4)
        if len(head) < 4:
            raise EOFError("end of file inside a record sequence")
        m = struct.unpack("<i", head)[0]
        size = abs(m)
        chunk = f.read(size)
        tail = f.read(4)
        if len(chunk) < size or len(tail) < 4:
            raise EOFError("truncated record")
        out.append(chunk)
        if m >= 0:
            return b"".join(out)


def _ints(b: bytes, n: int | None = None) -> tuple:
    v = struct.unpack(f"<{len(b) // 4}i", b)
    if n is not None and len(v) != n:
        raise ValueError(f"record holds {len(v)} integers, expected {n}")
    return v


def _i32(*vals) -> bytes:
    return struct.pack(f"<{len(vals)}i", *vals)


# ------------------------------------------------------------------ wave functions
def _band_host(psi, l: int) -> np.ndarray:
    """Band l of psi (numpy or torch, FP32/FP64, [M][N] x fastest) as real*8
    (the flat x-fastest order is Fortran's svecre(:,:,:) order)."""
    b = psi[l]
    if hasattr(b, "detach"):
        b = b.detach().to("cpu").numpy()
    return np.ascontiguousarray(b, dtype=np.float64).ravel()


def write_wf(directory: str, psi, sval: Sequence[float], shape, nr1: int = 0, nr2: int = 0,
             nrx: int = 0, nry: int = 0, nrz: int = 0, myr_kpt: int = 0,
             ksym: int = 0) -> str:
    """write_wf for a real (nrc = 0), non-magnetic (nums = ncol = 1), Gamma-only
    (numk = 1) set of bands psi[l] on the grid `shape` = (ncpx, ncpy, ncpz).
    Returns the path written."""
    ncpx, ncpy, ncpz = shape
    M = len(sval)
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, fname("wfc", nr1, nr2))
    with open(path, "wb") as f:
        write_record(f, _i32(WFC_VERSION))
        write_record(f, _i32(0, 1, 1, M, 1, ncpx, ncpy, ncpz))
        write_record(f, _i32(nrx, nry, nrz, myr_kpt))
        write_record(f, _i32(ksym))
        write_record(f, np.asarray(sval, dtype=np.float64))
        for l in range(M):
            write_record(f, _band_host(psi, l))
    return path


def read_wf(directory: str, neigmx: int, shape, out=None, nr1: int = 0, nr2: int = 0):
    """read_wf for the same layout as write_wf writes (real, nums = ncol = 1,
    numk = 1).  A file with more states than neigmx gives its first neigmx;
    fewer is an error, as in kukan.  Bands go into `out` ([neigmx][N], numpy
    or torch, any float type) when given, else into a new FP64 numpy array.
    Returns (sval, psi)."""
    ncpx, ncpy, ncpz = shape
    N = ncpx * ncpy * ncpz
    path = os.path.join(directory, fname("wfc", nr1, nr2))
    with open(path, "rb") as f:
        (ver,) = _ints(read_record(f), 1)
        if ver != WFC_VERSION:
            raise ValueError("wrong wfc version")
        nrc1, nums1, ncol1, neig1, numk1, cx, cy, cz = _ints(read_record(f), 8)
        read_record(f)  # nrx, nry, nrz, myr_kpt (not needed)
        read_record(f)  # ksym
        if (cx, cy, cz) != (ncpx, ncpy, ncpz) or nrc1 != 0 or nums1 != 1 or ncol1 != 1 \
                or numk1 != 1:
            raise ValueError(f"read_wf: unexpected array dimensions in file {path}")
        if neig1 < neigmx:
            raise ValueError(f"read_wf: not enough eigenstates in file {path}")
        sval1 = np.frombuffer(read_record(f), dtype="<f8")
        if out is None:
            out = np.empty((neigmx, N), dtype=np.float64)
        for l in range(neigmx):
            band = np.frombuffer(read_record(f), dtype="<f8")
            if band.size != N:
                raise ValueError("read_wf: band record of the wrong size")
            if hasattr(out, "copy_"):
                import torch
                out[l].copy_(torch.from_numpy(band.copy()).to(out.dtype))
            else:
                out[l] = band
    return sval1[:neigmx].copy(), out


# ------------------------------------------------------------------ densities, V_H
def write_rho(directory: str, rhosmt, shape, nr: int = 0, nrx: int = 0, nry: int = 0,
              nrz: int = 0, name: str = "rho", nradmx: int = 1, npoint: int = 1,
              natcell: Iterable[int] = (), rhotrur=None, rhosmtr=None) -> str:
    """write_rhovht's density file (nspv = 1).  Without PAW one-centre
    densities (rhotrur, rhosmtr None) no atom is listed and their records are
    empty, which read_rho accepts."""
    natcell = list(natcell)
    nat = len(natcell)
    ncpx, ncpy, ncpz = shape
    path = os.path.join(directory, fname(name, nr))
    os.makedirs(directory, exist_ok=True)
    rs = rhosmt.detach().to("cpu").numpy() if hasattr(rhosmt, "detach") else rhosmt
    g = np.ascontiguousarray(rs, dtype=np.float64).ravel()
    if g.size != ncpx * ncpy * ncpz:
        raise ValueError("write_rho: density of the wrong size")
    with open(path, "wb") as f:
        write_record(f, _i32(RHO_VERSION))
        write_record(f, _i32(1, ncpx, ncpy, ncpz, nradmx, npoint, nat))
        write_record(f, _i32(nrx, nry, nrz))
        write_record(f, _i32(nat, *natcell))
        write_record(f, g)
        for arr in (rhotrur, rhosmtr):
            write_record(f, b"" if arr is None else
                         np.asarray(arr, dtype=np.float64).reshape(nradmx, npoint, 1, nat,
                                                                   order="F"))
    return path


def read_rho(directory: str, shape, nr: int = 0, name: str = "rho"):
    """read_rho for nspv = 1: returns (rhosmt as a flat x-fastest FP64 array,
    natcell_inf, rhotrur, rhosmtr); None when the file does not exist
    (kukan then starts from the atomic density)."""
    ncpx, ncpy, ncpz = shape
    path = os.path.join(directory, fname(name, nr))
    if not os.path.exists(path):
        return None
    with open(path, "rb") as f:
        (ver,) = _ints(read_record(f), 1)
        if ver != RHO_VERSION:
            raise ValueError("wrong rho version")
        nspv1, cx, cy, cz, nradmx1, npoint1, nat1 = _ints(read_record(f), 7)
        read_record(f)
        info = _ints(read_record(f))
        if nspv1 != 1 or (cx, cy, cz) != (ncpx, ncpy, ncpz):
            raise ValueError(f"read_rho: unexpected array dimensions in density file {path}")
        na = info[0]
        natcell = list(info[1:1 + na])
        rho = np.frombuffer(read_record(f), dtype="<f8").copy()
        rt = np.frombuffer(read_record(f), dtype="<f8").reshape(nradmx1, npoint1, 1, nat1,
                                                                order="F")
        rs = np.frombuffer(read_record(f), dtype="<f8").reshape(nradmx1, npoint1, 1, nat1,
                                                                order="F")
    return rho, natcell, rt, rs


def write_vht(directory: str, vh_dense, shape, nmesh: int = 2, nr: int = 0, nrx: int = 0,
              nry: int = 0, nrz: int = 0) -> str:
    """write_rhovht's Hartree potential file (dense grid, x fastest)."""
    ncpx, ncpy, ncpz = shape
    path = os.path.join(directory, fname("vht", nr))
    os.makedirs(directory, exist_ok=True)
    v = vh_dense.detach().to("cpu").numpy() if hasattr(vh_dense, "detach") else vh_dense
    with open(path, "wb") as f:
        write_record(f, _i32(VHT_VERSION))
        write_record(f, _i32(ncpx, ncpy, ncpz, nmesh))
        write_record(f, _i32(nrx, nry, nrz))
        write_record(f, np.ascontiguousarray(v, dtype=np.float64).tobytes())
    return path


def read_vht(directory: str, shape, nmesh: int = 2, nr: int = 0):
    """read_vht: the dense V_H (flat, x fastest), or None without a file (kukan
    then starts the Hartree CG from zero)."""
    ncpx, ncpy, ncpz = shape
    path = os.path.join(directory, fname("vht", nr))
    if not os.path.exists(path):
        return None
    with open(path, "rb") as f:
        (ver,) = _ints(read_record(f), 1)
        if ver != VHT_VERSION:
            raise ValueError("wrong vht version")
        if _ints(read_record(f), 4) != (ncpx, ncpy, ncpz, nmesh):
            raise ValueError(f"read_vht: unexpected array dimensions in potential file {path}")
        read_record(f)
        v = np.frombuffer(read_record(f), dtype="<f8").copy()
    if v.size != ncpx * ncpy * ncpz * nmesh ** 3:
        raise ValueError("read_vht: potential record of the wrong size")
    return v
