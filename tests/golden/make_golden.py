"""Generates the analytic known-answer fixtures in this directory.

The reference ships no tests or outputs, so these vectors come from exact
mathematics, independent of both the oracle and the library:
  * fd_coefs.json: tools_definefdcoef's rationals (tools8f.F90:181-191) as
    fractions, and the plane-wave symbol of the nf=4 stencil;
  * poisson_fft.npz: the periodic FD Poisson problem -1/2 L v = 2 pi (rho -
    mean rho) on a small grid solved exactly in the DFT basis, where the
    discrete operator is diagonal (numpy.fft);
  * interp_trig.npz: coarse samples of a band-limited periodic function and
    its exact values on the dense (nmesh=2) points, for an error bound.
Run:  python tests/golden/make_golden.py
"""
import json
import os
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FD = {1: ["-2", "1"], 2: ["-5/2", "4/3", "-1/12"], 3: ["-49/18", "3/2", "-3/20", "1/90"],
      4: ["-205/72", "8/5", "-1/5", "8/315", "-1/560"],
      5: ["-36883/12600", "5/3", "-5/21", "5/126", "-5/1008", "1/3150"],
      6: ["-5369/1800", "12/7", "-15/56", "10/189", "-1/112", "2/1925", "-1/16632"]}


def central_second_derivative_weights(nf):
    """Exact Fornberg weights for d2/dx2 on offsets -nf..nf (rational)."""
    m = np.arange(-nf, nf + 1)
    A = [[Fraction(int(x)) ** k for x in m] for k in range(2 * nf + 1)]
    b = [Fraction(0)] * (2 * nf + 1)
    b[2] = Fraction(2)
    n = len(A)
    M = [row[:] + [b[i]] for i, row in enumerate(A)]
    for c in range(n):
        piv = next(r for r in range(c, n) if M[r][c] != 0)
        M[c], M[piv] = M[piv], M[c]
        for r in range(n):
            if r != c and M[r][c] != 0:
                f = M[r][c] / M[c][c]
                M[r] = [x - f * y for x, y in zip(M[r], M[c])]
    w = [M[i][n] / M[i][i] for i in range(n)]
    return [str(w[nf + k]) for k in range(nf + 1)]


def sym(n, h, a):
    k = np.arange(n)
    return -0.5 / h ** 2 * (a[0] + 2 * sum(a[m] * np.cos(2 * np.pi * k * m / n)
                                           for m in range(1, len(a))))


def main():
    out = {"fd": FD, "fornberg": {str(nf): central_second_derivative_weights(nf)
                                  for nf in range(1, 7)}}
    with open(os.path.join(HERE, "fd_coefs.json"), "w") as f:
        json.dump(out, f, indent=1)
    # Poisson
    nx, ny, nz = 16, 12, 20
    h = (0.41, 0.37, 0.33)
    rng = np.random.default_rng(7)
    rho = rng.standard_normal((nz, ny, nx))
    a = [float(Fraction(x)) for x in FD[4]]
    Lk = sym(nz, h[2], a)[:, None, None] + sym(ny, h[1], a)[None, :, None] + \
        sym(nx, h[0], a)[None, None, :]
    F = np.fft.fftn(rho - rho.mean())
    Lk[0, 0, 0] = 1.0
    V = 2 * np.pi * F / Lk
    V[0, 0, 0] = 0.0
    v = np.real(np.fft.ifftn(V))
    np.savez(os.path.join(HERE, "poisson_fft.npz"), shape=np.array([nx, ny, nz]), h=np.array(h),
             rho=rho.ravel(), v=v.ravel())
    # interpolation of a band-limited function
    nx, ny, nz = 12, 10, 14
    def f(x, y, z):
        return (np.cos(2 * np.pi * x) + 0.5 * np.sin(2 * np.pi * 2 * y) * np.cos(2 * np.pi * z)
                + 0.3 * np.sin(2 * np.pi * (x + z)))
    cz, cy, cx = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny,
                             (np.arange(nx) + 0.5) / nx, indexing="ij")
    dz, dy, dx = np.meshgrid((np.arange(2 * nz) + 0.5) / (2 * nz), (np.arange(2 * ny) + 0.5) /
                             (2 * ny), (np.arange(2 * nx) + 0.5) / (2 * nx), indexing="ij")
    np.savez(os.path.join(HERE, "interp_trig.npz"), shape=np.array([nx, ny, nz]),
             coarse=f(cx, cy, cz).ravel(), dense=f(dx, dy, dz).ravel())


if __name__ == "__main__":
    main()
