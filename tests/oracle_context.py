"""A stand-in for x3div_b200.Context on CPU tensors, for the multi-rank tests
over gloo: each routine and each pencil part of the step applies the oracle
along its direction on the given local extents (whole lines), so the pencil
code runs unchanged on host ranks.  Test infrastructure only."""
import socket

import numpy as np

KIND = {"derx": "der", "dery": "der", "derz": "der", "derxx": "der2", "deryy": "der2", "derzz": "der2",
        "derxvp": "dervp", "deryvp": "dervp", "derzvp": "dervp", "derxpv": "derpv", "derypv": "derpv",
        "derzpv": "derpv", "interxvp": "intvp", "interyvp": "intvp", "interzvp": "intvp",
        "interxpv": "intpv", "interypv": "intpv", "interzpv": "intpv"}


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleContext:
    """fused=False makes the pencil parts refuse (X3D_EUNSUPPORTED), as the
    library does for pencils its fused kernels cannot take, so that the
    pencil code composes them from the single-operator routines."""

    def __init__(self, oracle, shape, lengths, fused=True):
        self.o = oracle
        self.shape = shape
        self.lengths = lengths
        self.fused = fused
        self.d = [L / n for L, n in zip(lengths, shape)]

    def op(self, name):
        return name

    def _along(self, kind, d, a):
        import torch
        f = np.asfortranarray(a.numpy().transpose(2, 1, 0))
        r = self.o.apply(kind, d, f, self.d[d])
        return torch.from_numpy(np.ascontiguousarray(r.transpose(2, 1, 0)))

    def _refuse(self):
        if not self.fused:
            from x3div_b200._capi import X3D_EUNSUPPORTED
            from x3div_b200.api import X3DError
            raise X3DError(X3D_EUNSUPPORTED, "the stand-in's fused parts are off")

    def transeq_part(self, d, du, u, add, unew, dt, ext):
        self._refuse()
        vals = [self._along("der", d, u[d] * u[c]) + u[d] * self._along("der", d, u[c]) for c in range(3)]
        if add is not None:
            vals = [a + v for a, v in zip(add, vals)]
        for c in range(3):
            du[c].copy_(vals[c])
        if unew is not None:
            for c in range(3):
                unew[c].copy_(dt * du[c] + u[c])

    def divergence_part(self, d, out, ins, ext):
        self._refuse()
        if d == 0:
            res = [self._along("dervp", 0, ins[0]), self._along("intvp", 0, ins[1]),
                   self._along("intvp", 0, ins[2])]
        elif d == 1:
            res = [self._along("dervp", 1, ins[1]) + self._along("intvp", 1, ins[0]),
                   self._along("intvp", 1, ins[2])]
        else:
            res = [self._along("intvp", 2, ins[0]) + self._along("dervp", 2, ins[1])]
        for o, r in zip(out, res):
            o.copy_(r)

    def gradp_part(self, d, out, ins, ucor, ext):
        self._refuse()
        if d == 2:
            res = [self._along("intpv", 2, ins[0]), self._along("derpv", 2, ins[0])]
        elif d == 1:
            res = [self._along("intpv", 1, ins[0]), self._along("derpv", 1, ins[0]),
                   self._along("intpv", 1, ins[1])]
        else:
            res = [self._along("derpv", 0, ins[0]), self._along("intpv", 0, ins[1]),
                   self._along("intpv", 0, ins[2])]
        for o, r in zip(out, res):
            o.copy_(r)
        if ucor is not None:
            for c in range(3):
                ucor[c].sub_(out[c])

    def poisson_zpencil(self, spec, nxh_loc, i0, ny_loc, j0):
        """The z part of the spectral solve, restated with numpy's FFT and the
        oracle's modified-wavenumber tables, on a (nz, ny_loc, nxh_loc) block
        of x modes from i0 and y rows from j0."""
        import torch
        nx, ny, nz = self.shape
        t = self.o.poisson_tables(nx, ny, nz, *self.lengths)
        c = np.fft.fft(spec.numpy(), axis=0)
        i = (i0 + np.arange(nxh_loc))[None, None, :]
        j = (j0 + np.arange(ny_loc))[None, :, None]
        k = np.arange(nz)[:, None, None]
        tyz = t["ty"][j] * t["tz"][k]
        txz = t["tx"][i] * t["tz"][k]
        txy = t["tx"][i] * t["ty"][j]
        kk = t["k2x"][i] * tyz ** 2 + t["k2y"][j] * txz ** 2 + t["k2z"][k] * txy ** 2
        f = np.where(kk < 1e-16, 0.0, -1.0 / (np.where(kk < 1e-16, 1.0, kk) * (nx * ny * nz)))
        spec.copy_(torch.from_numpy(np.fft.ifft(c * f, axis=0) * nz))

    def __getattr__(self, routine):
        if routine not in KIND:
            raise AttributeError(routine)
        direction = "xyz".index(routine.replace("inter", "").replace("der", "")[0])

        def call(t, u, op, *extents):
            t.copy_(self._along(KIND[routine], direction, u))
        return call
