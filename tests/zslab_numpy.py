"""Test double of dft_b200.zslab.CudaSlabOps: the slab kernels' arithmetic in numpy on CPU
tensors, so that the z-slab driver's host logic (layouts, halo exchanges, reductions, the
replayed stop) runs on gloo ranks without a GPU.  numpy float64 operations round to nearest
without contraction, in the order written, which is the order of the CUDA kernels and of the
oracle (oracle/dft_oracle.c: hpsi3, oracle_hartree_potential_ex).  Test infrastructure only."""
import math

import numpy as np


def _spacing(grid):
    return grid.getDx(), grid.getDy(), grid.getDz()


class NumpySlabOps:
    def __init__(self, port=None):
        self.port = port

    def _port(self):
        if self.port is None:
            from oracle.bindings import Port
            self.port = Port()
        return self.port

    def jacobi_init(self, grid, z_lo, z_hi, Q, v, guess=None):
        nx, ny, nz = grid.nx, grid.ny, grid.nz
        dx, dy, dz = _spacing(grid)
        xmin, xmax, ymin, ymax, zmin, zmax = grid.bounds
        k = np.arange(z_lo, z_hi, dtype=np.int64)[:, None, None]
        j = np.arange(ny, dtype=np.int64)[None, :, None]
        i = np.arange(nx, dtype=np.int64)[None, None, :]
        shape = (z_hi - z_lo, ny, nx)
        x = np.broadcast_to(xmin + i.astype(np.float64) * dx, shape)
        y = np.broadcast_to(ymin + j.astype(np.float64) * dy, shape)
        z = np.broadcast_to(zmin + k.astype(np.float64) * dz, shape)
        face = np.broadcast_to((i == 0) | (i == nx - 1) | (j == 0) | (j == ny - 1) | (k == 0) | (k == nz - 1),
                               shape)
        d = [np.abs(x - xmin), np.abs(x - xmax), np.abs(y - ymin), np.abs(y - ymax),
             np.abs(z - zmin), np.abs(z - zmax)]
        m2 = np.minimum.reduce([q * q for q in d])
        r = np.sqrt(x * x + y * y + z * z)
        with np.errstate(divide="ignore", invalid="ignore"):
            bval = np.where((m2 > 0.0) & (r > 0.0), Q / r, 0.0)
        inner = guess.numpy().reshape(shape) if guess is not None else np.zeros(shape)
        v.numpy().reshape(shape)[...] = np.where(face, bval, inner)

    def jacobi_sweeps(self, grid, z_lo, z_hi, own_lo, own_hi, rho, v_in, v_out, scratch, sweeps, diffs):
        nx, ny = grid.nx, grid.ny
        nzl = z_hi - z_lo
        dx, dy, dz = _spacing(grid)
        ix, iy, iz = 1.0 / (dx * dx), 1.0 / (dy * dy), 1.0 / (dz * dz)
        den = 2.0 * (ix + iy + iz)
        c4pi = 4.0 * math.pi
        a = v_in.numpy().reshape(nzl, ny, nx)
        o = v_out.numpy().reshape(nzl, ny, nx)
        src = c4pi * rho.numpy().reshape(nzl, ny, nx)[1:-1, 1:-1, 1:-1]
        dv = diffs.numpy()
        dv[:sweeps] = 0.0
        o[...] = a
        # owned planes that the slab updates, as rows of the interior block
        lo, hi = max(own_lo - z_lo, 1) - 1, min(own_hi - z_lo, nzl - 1) - 1
        cur = a.copy()
        for t in range(sweeps):
            if nx >= 3 and ny >= 3 and nzl >= 3:
                c = cur[1:-1, 1:-1, 1:-1]
                sx = cur[1:-1, 1:-1, :-2] + cur[1:-1, 1:-1, 2:]
                sy = cur[1:-1, :-2, 1:-1] + cur[1:-1, 2:, 1:-1]
                sz = cur[:-2, 1:-1, 1:-1] + cur[2:, 1:-1, 1:-1]
                acc = ix * sx + iy * sy
                acc = acc + iz * sz
                acc = acc + src
                new = acc / den
                if hi > lo:
                    dv[t] = np.abs(new[lo:hi] - c[lo:hi]).max()
                nxt = cur.copy()
                nxt[1:-1, 1:-1, 1:-1] = new
                cur = nxt
        o[...] = cur
        scratch.numpy()[...] = np.nan  # the caller must not rely on it

    def hamiltonian(self, grid, z_lo, z_hi, V, psi, hpsi, nbands):
        nx, ny = grid.nx, grid.ny
        nzl = z_hi - z_lo
        dx, dy, dz = _spacing(grid)
        ix, iy, iz = 1.0 / (dx * dx), 1.0 / (dy * dy), 1.0 / (dz * dz)
        P = psi.numpy().reshape(nbands, nzl, ny, nx)
        W = V.numpy().reshape(1, nzl, ny, nx)
        lap = (-2.0 * (ix + iy + iz)) * P
        lap[..., 1:] = lap[..., 1:] + P[..., :-1] * ix
        lap[..., :-1] = lap[..., :-1] + P[..., 1:] * ix
        lap[..., 1:, :] = lap[..., 1:, :] + P[..., :-1, :] * iy
        lap[..., :-1, :] = lap[..., :-1, :] + P[..., 1:, :] * iy
        lap[:, 1:] = lap[:, 1:] + P[:, :-1] * iz
        lap[:, :-1] = lap[:, :-1] + P[:, 1:] * iz
        hpsi.numpy().reshape(nbands, nzl, ny, nx)[...] = -0.5 * lap + W * P

    # ---- XC and Gram: the oracle's functional on the slab, numpy reductions ----------------
    def xc(self, grid, z_lo, z_hi, own_lo, own_hi, kind, na, nb, va, vb):
        port = self._port()
        nx, ny = grid.nx, grid.ny
        nzl = z_hi - z_lo
        dx, dy, dz = _spacing(grid)
        xmin, xmax, ymin, ymax, zmin, _ = grid.bounds
        a, b = na.numpy(), nb.numpy()
        # the slab as its own grid: the same spacing up to rounding of its bounds
        sb = (xmin, xmax, ymin, ymax, zmin + z_lo * dz, zmin + (z_hi - 1) * dz)
        if va is not None:
            va.numpy()[...] = port.xc_potential(kind, (nx, ny, nzl), sb, a, b, 0)
        if vb is not None:
            vb.numpy()[...] = port.xc_potential(kind, (nx, ny, nzl), sb, a, b, 1)

        def gradmag(f):
            f3 = f.reshape(nzl, ny, nx)
            out = []
            for axis, h in ((2, dx), (1, dy), (0, dz)):
                g = np.empty_like(f3)
                sl = [slice(None)] * 3

                def at(s):
                    q = list(sl)
                    q[axis] = s
                    return tuple(q)
                g[at(slice(1, -1))] = (f3[at(slice(2, None))] - f3[at(slice(None, -2))]) / (2.0 * h)
                g[at(0)] = (f3[at(1)] - f3[at(0)]) / h
                g[at(-1)] = (f3[at(-1)] - f3[at(-2)]) / h
                out.append(g)
            return np.sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]).ravel()

        n_xy = nx * ny
        lo, hi = (own_lo - z_lo) * n_xy, (own_hi - z_lo) * n_xy
        ga, gb = gradmag(a)[lo:hi], gradmag(b)[lo:hi]
        oa, ob = a[lo:hi], b[lo:hi]
        eps = port.xc_evaluate(kind, oa, ob, ga, gb)[:, 0]
        n = oa + ob
        keep = n > 1.0e-20
        return float(np.sum(n[keep] * eps[keep]) * (dx * dy * dz))

    def gram(self, grid, z_lo, z_hi, own_lo, own_hi, A, ka, B, kb, precision=0):
        import torch
        n_xy = grid.nx * grid.ny
        lo, hi = (own_lo - z_lo) * n_xy, (own_hi - z_lo) * n_xy
        a = A.numpy().reshape(ka, -1)[:, lo:hi]
        b = B.numpy().reshape(kb, -1)[:, lo:hi]
        dx, dy, dz = _spacing(grid)
        return torch.from_numpy((a @ b.T) * (dx * dy * dz))
