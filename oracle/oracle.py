"""ctypes front end of the CPU oracle (oracle/rs_oracle*.c).

TEST INFRASTRUCTURE ONLY.  tests/, ``__graft_entry__.smoke()`` and the CPU
legs of ``bench.py`` import this module as the checker; the product package
``rspacedist_b200`` never does.  Every function takes and returns numpy arrays
in the layouts documented in ``rs_oracle.h``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "librs_oracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off); make
    rebuilds only when a source is newer than the library."""
    if force and os.path.exists(_SO):
        os.remove(_SO)
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_SO)
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class OrcSys(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nf", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("N", C.c_long),
        ("natom", C.c_int), ("nprjmx", C.c_int), ("num_list", C.c_int),
        ("nprj", _ip), ("natinf", _ip), ("lst", _ip),
        ("v", _dp), ("dij", _dp), ("sss", _dp), ("veff", _dp),
    ]


class OrcPrm(C.Structure):
    _fields_ = [
        ("northo", C.c_int), ("nsdmax", C.c_int), ("nprecon", C.c_int),
        ("epssd", C.c_double),
        ("ndiismax", C.c_int),
        ("eps_eig_diis", C.c_double), ("alambda_diis", C.c_double),
        ("alambda_min", C.c_double), ("alambda_max", C.c_double),
    ]


def fdcoef(nf):
    a = np.zeros(9)
    lib().orc_fdcoef(C.c_int(nf), _d(a))
    return a


def tree_dot(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    L = lib()
    if a.dtype == np.float32:
        L.orc_tree_dot_f.restype = C.c_double
        return L.orc_tree_dot_f(C.c_long(a.size), a.ctypes.data_as(_fp), b.ctypes.data_as(_fp))
    L.orc_tree_dot.restype = C.c_double
    return L.orc_tree_dot(C.c_long(a.size), _d(_f64(a)), _d(_f64(b)))


def kslaplacian(shape, nf, h, psi, veff, out=None):
    nx, ny, nz = shape
    psi = _f64(psi)
    nb = psi.size // (nx * ny * nz)
    out = np.zeros_like(psi) if out is None else _f64(out).copy()
    lib().orc_kslaplacian(nx, ny, nz, nf, C.c_double(h[0]), C.c_double(h[1]), C.c_double(h[2]),
                          _d(psi), _d(_f64(veff)), _d(out), nb)
    return out


def precondition(shape, x):
    nx, ny, nz = shape
    x = _f64(x)
    out = np.empty_like(x)
    lib().orc_precondition(nx, ny, nz, _d(x), _d(out), x.size // (nx * ny * nz))
    return out


def nl_dot(geo, psi, N):
    psi = _f64(psi)
    nb = psi.size // N
    rp = np.zeros((nb, geo["natom"], geo["nprjmx"]))
    lib().orc_nl_dot(geo["natom"], geo["nprjmx"], geo["num_list"], _i(geo["nprj"]),
                     _i(geo["natinf"]), _i(geo["lst"]), _d(geo["v"]), _d(psi), C.c_long(N), nb,
                     _d(rp))
    return rp


def nl_apply(geo, mat, dvol, rp, N, out):
    out = _f64(out).copy()
    rp = _f64(rp)
    nb = out.size // N
    lib().orc_nl_apply(geo["natom"], geo["nprjmx"], geo["num_list"], _i(geo["nprj"]),
                       _i(geo["natinf"]), _i(geo["lst"]), _d(geo["v"]), _d(_f64(mat)),
                       C.c_double(dvol), _d(rp), C.c_long(N), nb, _d(out))
    return out


def make_sys(geo, shape, nf, h, veff, dij, sss=None):
    """Build an OrcSys; the returned tuple keeps the numpy buffers alive."""
    keep = dict(nprj=_i32(geo["nprj"]), natinf=_i32(geo["natinf"]), lst=_i32(geo["lst"]),
                v=_f64(geo["v"]), dij=_f64(dij), veff=_f64(veff))
    if sss is not None:
        keep["sss"] = _f64(sss)
    s = OrcSys()
    s.nx, s.ny, s.nz = shape
    s.nf = nf
    s.dx, s.dy, s.dz = h
    s.N = shape[0] * shape[1] * shape[2]
    s.natom, s.nprjmx, s.num_list = geo["natom"], geo["nprjmx"], geo["num_list"]
    s.nprj, s.natinf, s.lst = _i(keep["nprj"]), _i(keep["natinf"]), _i(keep["lst"])
    s.v, s.dij, s.veff = _d(keep["v"]), _d(keep["dij"]), _d(keep["veff"])
    s.sss = _d(keep["sss"]) if sss is not None else C.cast(None, _dp)
    return s, keep


def hpsi(sysk, psi, rp):
    s, _ = sysk
    psi = _f64(psi)
    nb = psi.size // s.N
    out = np.empty_like(psi)
    lib().orc_apply_h(C.byref(s), _d(psi), _d(_f64(rp)), _d(out), nb)
    return out


def spsi(sysk, psi, rp):
    s, _ = sysk
    psi = _f64(psi)
    nb = psi.size // s.N
    out = np.empty_like(psi)
    lib().orc_apply_s(C.byref(s), _d(psi), _d(_f64(rp)), _d(out), nb)
    return out


def hpsi_fast(sysk, psi, rp, nthreads):
    s, _ = sysk
    psi = _f64(psi)
    nb = psi.size // s.N
    out = np.empty_like(psi)
    lib().orc_hpsi_fast(C.byref(s), _d(psi), _d(_f64(rp)), _d(out), nb, nthreads)
    return out


def density(occ, psi, N):
    psi = _f64(psi)
    rho = np.zeros(N)
    lib().orc_density(C.c_long(N), psi.size // N, _d(_f64(occ)), _d(psi), _d(rho))
    return rho


def interp_c2d(shape, nf, x):
    nx, ny, nz = shape
    out = np.zeros(8 * nx * ny * nz)
    lib().orc_interp_c2d(nx, ny, nz, nf, _d(_f64(x)), _d(out))
    return out


def interp_d2c(shape, nf, x):
    """Dense (2nx, 2ny, 2nz) -> coarse (nx, ny, nz) transfer (trans_d2c_*)."""
    nx, ny, nz = shape
    out = np.zeros(nx * ny * nz)
    lib().orc_interp_d2c(nx, ny, nz, nf, _d(_f64(x)), _d(out))
    return out


def vxc_pz(rho):
    rho = _f64(rho)
    vx, ex = np.zeros(rho.size), np.zeros(rho.size)
    lib().orc_vxc_pz(C.c_long(rho.size), _d(rho), _d(vx), _d(ex))
    return vx, ex


def veff_sum(vx, vloc, vh):
    vx = _f64(vx)
    out = np.zeros(vx.size)
    lib().orc_veff_sum(C.c_long(vx.size), _d(vx), _d(_f64(vloc)), _d(_f64(vh)), _d(out))
    return out


def diffcharge(rho_o, rho_i, h, xmax):
    L = lib()
    L.orc_diffcharge.restype = C.c_double
    rho_o = _f64(rho_o)
    return L.orc_diffcharge(C.c_long(rho_o.size), _d(rho_o), _d(_f64(rho_i)),
                            *(C.c_double(v) for v in h), *(C.c_double(v) for v in xmax))


def atomicocc(nprj, nprjmx, rp, fnele):
    """scf_charge_atomicocc: rp [M][natom][nprjmx], fnele [M] ->
    atocc [natom][nprjmx (nprjmx+1) / 2] (packed upper triangle, j outer)."""
    L = lib()
    nprj = np.ascontiguousarray(nprj, np.int32)
    natom = nprj.size
    rp = _f64(rp)
    fnele = _f64(fnele)
    M = fnele.size
    out = np.zeros((natom, nprjmx * (nprjmx + 1) // 2))
    L.orc_atomicocc(natom, nprjmx, _i(nprj), M, _d(rp), _d(fnele), _d(out))
    return out


class Broyden:
    """scf_chargemixing with modified Broyden history (one spin, grid density)."""

    def __init__(self, n, nbrydn=20, eta=0.02):
        L = lib()
        L.orc_broyden_create.restype = C.c_void_p
        self.h = C.c_void_p(L.orc_broyden_create(C.c_long(n), nbrydn, C.c_double(eta)))
        self.n = n

    def step(self, rho_o, rho_i, dvol):
        """Returns the next input density (rho_i is not modified)."""
        r = _f64(rho_i).copy()
        lib().orc_broyden_step(self.h, _d(_f64(rho_o)), _d(r), C.c_double(dvol))
        return r

    def __del__(self):
        try:
            lib().orc_broyden_free(self.h)
        except Exception:
            pass


def hartree_laplacian(shape, nfh, h, v):
    nx, ny, nz = shape
    out = np.zeros(nx * ny * nz)
    lib().orc_hartree_laplacian(nx, ny, nz, nfh, C.c_double(h[0]), C.c_double(h[1]),
                                C.c_double(h[2]), _d(_f64(v)), _d(out))
    return out


def hartree_cg(shape, nfh, xmax, epsvh, ncgmin, ncgmax, ncgres, rho, vh0):
    nx, ny, nz = shape
    vh = _f64(vh0).copy()
    dp = C.c_double(0)
    it = lib().orc_hartree_cg(nx, ny, nz, nfh, C.c_double(xmax[0]), C.c_double(xmax[1]),
                              C.c_double(xmax[2]), C.c_double(epsvh), ncgmin, ncgmax, ncgres,
                              _d(_f64(rho)), _d(vh), C.byref(dp))
    return vh, it, dp.value


def gradient(shape, nf, h, axis, psi):
    nx, ny, nz = shape
    out = np.zeros(nx * ny * nz)
    lib().orc_gradient(nx, ny, nz, nf, C.c_double(h), axis, _d(_f64(psi)), _d(out))
    return out


def sphere_lists(atoms, rcut, nmax, h, npmax, nfdg, num_list):
    atoms = _f64(atoms).reshape(-1, 3)
    A = atoms.shape[0]
    ax, ay, az = (np.ascontiguousarray(atoms[:, k]) for k in range(3))
    rc = _f64(np.broadcast_to(rcut, (A,)))
    nat = [np.zeros(A, np.int32) for _ in range(3)]
    natinf = np.zeros(A, np.int32)
    lst = np.zeros(A * num_list, np.int32)
    lx, ly, lz = (np.zeros(A * num_list, np.int32) for _ in range(3))
    st = lib().orc_sphere_lists(A, _d(ax), _d(ay), _d(az), _d(rc), nmax[0], nmax[1], nmax[2],
                                C.c_double(h[0]), C.c_double(h[1]), C.c_double(h[2]),
                                npmax[0], npmax[1], npmax[2], nfdg, num_list,
                                _i(nat[0]), _i(nat[1]), _i(nat[2]), _i(natinf), _i(lst),
                                _i(lx), _i(ly), _i(lz))
    return st, dict(natx=nat[0], naty=nat[1], natz=nat[2], natinf=natinf, lst=lst,
                    lstx=lx, lsty=ly, lstz=lz)


def jacobi_eig(a):
    a = _f64(a).copy()
    n = a.shape[0]
    w = np.zeros(n)
    z = np.zeros((n, n))
    st = lib().orc_jacobi_eig(n, _d(a), _d(w), _d(z))
    return st, w, z


def eig2(a):
    a = _f64(a).reshape(4).copy()
    w = np.zeros(2)
    z = np.zeros(4)
    lib().orc_eig2(_d(a), _d(w), _d(z))
    return w, z.reshape(2, 2)


def reorder_rank(sval):
    r = np.zeros(len(sval), np.int32)
    lib().orc_reorder_rank(len(sval), _d(_f64(sval)), _i(r))
    return r


def ortho(sysk, M, psi, spsi, rp, l_inp=0, cmpt=1):
    s, _ = sysk
    psi = _f64(psi).copy()
    rp = _f64(rp).copy()
    if spsi is None:
        lib().orc_ortho(C.byref(s), M, l_inp, cmpt, _d(psi), _d(psi), _d(rp))
        return psi, None, rp
    spsi = _f64(spsi).copy()
    lib().orc_ortho(C.byref(s), M, l_inp, cmpt, _d(psi), _d(spsi), _d(rp))
    return psi, spsi, rp


def rayleighritz(sysk, M, psi, spsi, rp):
    s, _ = sysk
    psi = _f64(psi).copy()
    rp = _f64(rp).copy()
    h = np.zeros_like(psi)
    sval = np.zeros(M)
    sp = psi if spsi is None else _f64(spsi).copy()
    st = lib().orc_rayleighritz(C.byref(s), M, 1, _d(psi), _d(sp), _d(rp), _d(h), _d(sval))
    return st, psi, (None if spsi is None else sp), rp, sval


def _prm(northo=1, nsdmax=4, nprecon=1, epssd=1e-6, ndiismax=4, eps_eig_diis=1e-14,
         alambda_diis=0.5, alambda_min=0.1, alambda_max=1.0):
    p = OrcPrm()
    p.northo, p.nsdmax, p.nprecon, p.epssd = northo, nsdmax, nprecon, epssd
    p.ndiismax, p.eps_eig_diis = ndiismax, eps_eig_diis
    p.alambda_diis, p.alambda_min, p.alambda_max = alambda_diis, alambda_min, alambda_max
    return p


def kscg(sysk, M, psi, spsi, rp, **prm):
    s, _ = sysk
    p = _prm(**prm)
    psi = _f64(psi).copy()
    rp = _f64(rp).copy()
    sp = psi if spsi is None else _f64(spsi).copy()
    h = np.zeros_like(psi)
    sval = np.zeros(M)
    resid = np.zeros(M)
    itm = C.c_int(0)
    st = lib().orc_kscg(C.byref(s), C.byref(p), M, _d(psi), _d(sp), _d(rp), _d(h), _d(sval),
                        _d(resid), C.byref(itm))
    return st, psi, (None if spsi is None else sp), rp, h, sval, resid


def ksdiis(sysk, M, psi, spsi, rp, l_hsv=1, **prm):
    s, _ = sysk
    p = _prm(**prm)
    psi = _f64(psi).copy()
    rp = _f64(rp).copy()
    sp = psi if spsi is None else _f64(spsi).copy()
    h = np.zeros_like(psi)
    sval = np.zeros(M)
    resid = np.zeros(M)
    conv = lib().orc_ksdiis(C.byref(s), C.byref(p), M, l_hsv, _d(psi), _d(sp), _d(rp), _d(h),
                            _d(sval), _d(resid))
    return conv, psi, (None if spsi is None else sp), rp, h, sval, resid


def force_nl(sysk, M, psi, sval, occ):
    s, _ = sysk
    A = s.natom
    fx, fy, fz = np.zeros(A), np.zeros(A), np.zeros(A)
    lib().orc_force_nl(C.byref(s), M, _d(_f64(psi)), _d(_f64(sval)), _d(_f64(occ)), _d(fx),
                       _d(fy), _d(fz))
    return np.stack([fx, fy, fz], axis=1)


def dg_weights(nfdg, npmesh):
    """wxyz of pseudocalc_01a, index j + nfdg*npmesh."""
    w = np.zeros(2 * nfdg * npmesh)
    lib().orc_dg_weights(nfdg, npmesh, _d(w))
    return w


def projector_tables(atoms, lists, nmax, h, npmax, nfdg, npmesh, num_list, prj_col, prj_m,
                     coef, nqct, nqmx, rcut, psftrad, psctoff, eps, nfiltyp, filpp, wxyz):
    """vnlocp (natom, nprj, num_list) of pseudocalc_07 for one species; lists
    is the dict returned by sphere_lists (natx.., natinf, lstx..)."""
    atoms = _f64(atoms).reshape(-1, 3)
    A = atoms.shape[0]
    ax, ay, az = (np.ascontiguousarray(atoms[:, k]) for k in range(3))
    ii = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    col, ym = ii(prj_col), ii(prj_m)
    P = len(col)
    v = np.zeros((A, P, num_list))
    keep = [ii(lists[k]) for k in ("natx", "naty", "natz", "natinf", "lstx", "lsty", "lstz")]
    st = lib().orc_projector_tables(
        A, P, num_list, nmax[0], nmax[1], nmax[2], C.c_double(h[0]), C.c_double(h[1]),
        C.c_double(h[2]), npmax[0], npmax[1], npmax[2], nfdg, npmesh, _d(ax), _d(ay), _d(az),
        *[_i(k) for k in keep], _i(col), _i(ym), nqct, nqmx, _d(_f64(coef)), C.c_double(rcut),
        C.c_double(psftrad), C.c_double(psctoff), C.c_double(eps), nfiltyp, C.c_double(filpp),
        _d(_f64(wxyz)), _d(v))
    assert st == 0, "orc_projector_tables: out of memory"
    return v


# ---- local pseudopotential, Ewald energy, initial bands (rs_oracle_vloc.c) ----

def bisec(z, r, eps=1.0e-12):
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    lib().orc_bisec(C.c_double(z), C.c_double(r), C.c_double(eps), C.byref(a), C.byref(b),
                    C.byref(c))
    return a.value, b.value, c.value


def vloc_coef(radial, dradial, potc, nradct, a, b, c, rcuts, nqct):
    radial, dradial, potc = _f64(radial), _f64(dradial), _f64(potc)
    coef = np.zeros(nqct + 1)
    lib().orc_vloc_coef(len(radial), nradct, _d(radial), _d(dradial), _d(potc), C.c_double(a),
                        C.c_double(b), C.c_double(c), C.c_double(rcuts), nqct, _d(coef))
    return coef


def vloc_soft(atoms, cp1, a, b, c, rc, shape, h, xmax, veta, npw, grad=False):
    atoms = _f64(atoms).reshape(-1, 3)
    A = atoms.shape[0]
    ax, ay, az = (np.ascontiguousarray(atoms[:, k]) for k in range(3))
    N = int(np.prod(shape))
    out = np.zeros(N)
    g = np.zeros(3 * A * N) if grad else None
    f = C.c_double
    lib().orc_vloc_soft(A, _d(ax), _d(ay), _d(az), f(cp1), f(a), f(b), f(c), f(rc), shape[0],
                        shape[1], shape[2], f(h[0]), f(h[1]), f(h[2]), f(xmax[0]), f(xmax[1]),
                        f(xmax[2]), f(veta), npw[0], npw[1], npw[2], _d(out),
                        _d(g) if grad else None)
    return (out, g.reshape(3, A, N)) if grad else out


def vloc_hard(atoms, nmax, nmesh, h, xmax, npmax, rcut, psctoff, rcuts, nqct, coef, filpp, eps,
              nfiltyp, dense=None, rho_dense=None):
    """Adds each atom's hard part to dense (8N for nmesh 2, modified in place
    when given); with rho_dense returns the per-atom sums of rho times the
    hard part's gradient times the dense volume element (natom x 3)."""
    atoms = _f64(atoms).reshape(-1, 3)
    A = atoms.shape[0]
    ax, ay, az = (np.ascontiguousarray(atoms[:, k]) for k in range(3))
    f = C.c_double
    facc = np.zeros(3 * A) if rho_dense is not None else None
    rd = _f64(rho_dense) if rho_dense is not None else None
    lib().orc_vloc_hard(A, _d(ax), _d(ay), _d(az), nmax[0], nmax[1], nmax[2], nmesh, f(h[0]),
                        f(h[1]), f(h[2]), f(xmax[0]), f(xmax[1]), f(xmax[2]), npmax[0], npmax[1],
                        npmax[2], f(rcut), f(psctoff), f(rcuts), nqct, _d(_f64(coef)), f(filpp),
                        f(eps), nfiltyp, _d(dense) if dense is not None else None,
                        _d(rd) if rd is not None else None,
                        _d(facc) if facc is not None else None)
    return facc.reshape(A, 3) if facc is not None else dense


def ewald(atoms, cp1, xmax, veta, npw, nrs):
    atoms = _f64(atoms).reshape(-1, 3)
    ax, ay, az = (np.ascontiguousarray(atoms[:, k]) for k in range(3))
    fn = lib().orc_ewald
    fn.restype = C.c_double
    f = C.c_double
    return fn(atoms.shape[0], _d(ax), _d(ay), _d(az), f(cp1), f(xmax[0]), f(xmax[1]),
              f(xmax[2]), f(veta), npw[0], npw[1], npw[2], nrs[0], nrs[1], nrs[2])


def initial_wave(atoms, cp1, zs_pre, neig, shape, h, xmax):
    atoms = _f64(atoms).reshape(-1, 3)
    ax, ay, az = (np.ascontiguousarray(atoms[:, k]) for k in range(3))
    N = int(np.prod(shape))
    psi = np.zeros(neig * N)
    f = C.c_double
    lib().orc_initial_wave(atoms.shape[0], _d(ax), _d(ay), _d(az), f(cp1), f(zs_pre), neig,
                           shape[0], shape[1], shape[2], f(h[0]), f(h[1]), f(h[2]), f(xmax[0]),
                           f(xmax[1]), f(xmax[2]), _d(psi))
    return psi.reshape(neig, N)
