"""Derives the compact pseudopotential tables in this directory from RSPACE's
dataset files (read where the reference tree is mounted; the generated JSON is
what the package loads).

    python -m rspacedist_b200.data.make_pp_tables /path/to/RSPACEes.v08.01

For each dataset it keeps what the real-space hot path consumes:
  * the projector radial functions p_{l,i}(r) = (r p)(r) / r of every dyadic
    present (the reader's loop at read_ppfile8f.F90:197-209), resampled with
    cubic interpolation on a uniform radial grid of step 0.005 bohr up to the
    last mesh point nradct;
  * the charge-deficit matrix qvd (sss0, :213-217) and dion (akv0, in Ry,
    halved to Ha as at :221-225) over the dyadic slots;
  * the cut-off radius radial(nradct), the valence charge and the short-range
    local potential potc = (vloc - vh)/2 in Ha (:160-167) on the same grid;
  * the dataset's own radial mesh r, dr/di (nradps points, nradct of them
    inside the cut-off), potc on that mesh and, for PAW datasets, the density
    column the reader feeds to the LDA before subtracting v_xc from potc
    (:158-186): the local pseudopotential's Fourier-Bessel coefficients are
    summed over this mesh as filterpseudopotentials does.
"""
import json
import os
import sys

import numpy as np
from scipy.interpolate import CubicSpline

DATASETS = {"si_paw": "PAW/paw.014", "c_ncps": "NCPS/paw.006"}
DR = 0.005


def parse(path):
    with open(path) as f:
        lines = f.read().splitlines()
    it = iter(lines)
    nxt = lambda: next(it)
    for _ in range(11):
        nxt()
    kind = nxt().strip().lower()
    nxt()
    z, zv = (float(x) for x in nxt().split()[:2])
    nxt()
    lmax = int(nxt().split()[0]) - 1
    nxt()
    nprmx = int(nxt().split()[0])
    nxt()
    npr = []
    for l in range(lmax + 1):
        npr.append(int(nxt().split()[1]))
    nxt(); nxt(); nxt(); nxt()
    for _ in range(6):
        nxt()
    nxt()
    nradps, nradct = (int(x) for x in nxt().split()[:2])
    nxt()
    mesh = np.array([[float(x) for x in nxt().split()] for _ in range(nradps)])
    nxt()
    nxt()
    for _ in range(nradps):
        nxt()
    nxt()
    nrprj = nprmx * (lmax + 1)
    prj = np.zeros((nrprj, nradct))
    for j in range(nrprj):
        nxt(); nxt(); nxt()
        for ir in range(nradct):
            prj[j, ir] = float(nxt().split()[2])
    nxt(); nxt()
    qvd = np.array([[float(x) for x in nxt().split()] for _ in range(nrprj)])
    nxt(); nxt()
    dion = np.array([[float(x) for x in nxt().split()] for _ in range(nrprj)]) * 0.5
    return dict(kind=kind, z=z, zv=zv, lmax=lmax, nprmx=nprmx, npr=npr, mesh=mesh,
                nradps=nradps, nradct=nradct, prj=prj, qvd=qvd, dion=dion)


def derive(d):
    r = d["mesh"][: d["nradct"], 0]
    rc = float(r[-1])
    grid = np.arange(0.0, rc + 1e-12, DR)
    out = dict(kind=d["kind"], z=d["z"], zv=d["zv"], lmax=d["lmax"], nprmx=d["nprmx"],
               npr=d["npr"], rcut=rc, dr=DR, channels=[])
    for l in range(d["lmax"] + 1):
        for i in range(d["npr"][l]):
            slot = l * d["nprmx"] + i
            rp = d["prj"][slot]
            p = np.where(r > 1e-8, rp / np.maximum(r, 1e-300), 0.0)
            # value at r=0 by extrapolation from the first positive points
            p[0] = p[1] + (p[1] - p[2]) * (r[1] - r[0]) / (r[2] - r[1]) if l == 0 else 0.0
            cs = CubicSpline(r, p)
            out["channels"].append(dict(l=l, i=i, slot=slot, p=[float(x) for x in cs(grid)]))
    out["qvd"] = d["qvd"].tolist()
    out["dion_ha"] = d["dion"].tolist()
    m = d["mesh"]
    potc = (m[:, 2] - m[:, 4]) * 0.5
    sel = m[:, 0] > 0
    cs = CubicSpline(m[sel, 0], potc[sel])
    rr = np.arange(DR, min(12.0, m[sel, 0].max()), DR)
    out["potc_dr"] = DR
    out["potc"] = [float(cs(DR))] + [float(x) for x in cs(rr)]
    out["nradps"] = int(d["nradps"])
    out["nradct"] = int(d["nradct"])
    out["mesh_r"] = [float(x) for x in m[:, 0]]
    out["mesh_drdi"] = [float(x) for x in m[:, 1]]
    out["mesh_potc"] = [float(x) for x in potc]
    out["mesh_rho"] = [float(x) for x in m[:, 6]]
    return out


def main(root):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, rel in DATASETS.items():
        d = derive(parse(os.path.join(root, rel)))
        with open(os.path.join(here, name + ".json"), "w") as f:
            json.dump(d, f)
        print(name, d["kind"], "rcut", d["rcut"], "channels",
              [(c["l"], c["i"]) for c in d["channels"]])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m rspacedist_b200.data.make_pp_tables <RSPACEes.v08.01 directory>")
    main(sys.argv[1])
