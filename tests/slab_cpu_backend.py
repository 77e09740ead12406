"""A CPU rank for cola_halo_b200.slab.SlabPM: the same stages as the
library's cg_sim_slab_* (deposit and r2c along z of a slab of planes, the
x / Green / inverse x passes of a slab of kz planes, the z c2r and the
interpolation of a slab), in numpy float64 on full-size meshes, with the
spectra held in float32 CPU tensors like the device's.  Test infrastructure
only: it lets the decomposition's exchanges (buffer particles, transposes,
particle moves) run as gloo ranks on CPU and be checked against the
oracle's undivided force (oracle/restate.py: pm_calculate_forces)."""
import math

import numpy as np
import torch

from oracle import restate as R

f32 = np.float32


class CpuRank:
    def __init__(self, ngrid, boxsize, factor, rows):
        self.N, self.L, self.factor = ngrid, float(boxsize), factor
        self.rows = rows.clone()                       # n x 14 float32 (reference Particle)
        self.f = torch.zeros((3, self.n), dtype=torch.float32)
        H1 = ngrid // 2 + 1
        self.spec = [torch.zeros((H1, ngrid, ngrid, 2), dtype=torch.float32) for _ in range(4)]
        self.meshes = [np.zeros((ngrid,) * 3) for _ in range(3)]

    @property
    def n(self):
        return self.rows.shape[0]

    def sync(self):
        pass

    def positions(self):
        return self.rows[:, :3].T

    def forces(self):
        return self.f

    def spectrum(self, which):
        return self.spec[which]

    def get_particles(self):
        return self.rows.clone()

    def set_particles(self, rows):
        self.rows = rows.clone()
        self.f = torch.zeros((3, self.n), dtype=torch.float32)

    # -- stages
    def _deposit(self, mesh, pos, x0, nx):
        N = self.N
        if len(pos) == 0:
            return
        iI, I1, J, J1, K, K1, D1, D2, D3, T1, T2, T3 = R._cic_index(pos, N, self.L)
        w = f32(f32(self.factor) ** 3)
        for ix, wx in ((iI, T1), (I1, D1)):
            own = (ix >= x0) & (ix < x0 + nx)
            for jy, wy in ((J, T2), (J1, D2)):
                for kz, wz in ((K, T3), (K1, D3)):
                    v = wx.astype(np.float64) * wy * wz * w
                    np.add.at(mesh, (ix[own], jy[own], kz[own]), v[own])

    def density(self, x0, nx, bx):
        N = self.N
        mesh = np.zeros((N, N, N))
        mesh[x0:x0 + nx] = -1.0
        self._deposit(mesh, self.rows[:, :3].numpy(), x0, nx)
        self._deposit(mesh, bx.T.numpy(), x0, nx)
        zk = np.fft.rfft(mesh[x0:x0 + nx], axis=2)          # [x][y][kz]
        s = self.spec[0]
        t = np.transpose(zk, (2, 0, 1))                       # [kz][x][y]
        s[:, x0:x0 + nx, :, 0] = torch.from_numpy(t.real.astype(f32))
        s[:, x0:x0 + nx, :, 1] = torch.from_numpy(t.imag.astype(f32))
        return float(mesh[x0:x0 + nx].sum())

    def kspace(self, kz0, nkz):
        N = self.N
        s = self.spec[0][kz0:kz0 + nkz].numpy()
        d = s[..., 0].astype(np.float64) + 1j * s[..., 1]
        dk = np.fft.fft(np.fft.fft(d, axis=1), axis=2)        # [kz][kx][ky]
        scale = f32(2.0 * math.pi / np.float64(f32(self.L)))
        f1 = f32(-1.0 / N ** 3 / np.float64(scale))
        idx = np.arange(N)
        sg = np.where(idx <= N // 2, idx, idx - N)
        K = np.arange(kz0, kz0 + nkz)[:, None, None]
        I0 = sg[None, :, None]
        J0 = sg[None, None, :]
        den = K * K + I0 * I0 + J0 * J0
        g = (f1 / np.where(den == 0, 1, den).astype(f32)).astype(f32)
        for a, n_a in enumerate((I0, J0, K)):
            f2 = (g * np.asarray(n_a, dtype=f32)).astype(f32).astype(np.float64)
            F = 1j * f2 * dk
            F[den == 0] = 0.0
            G = np.fft.ifft(np.fft.ifft(F, axis=2), axis=1) * (N * N)
            t = self.spec[1 + a]
            t[kz0:kz0 + nkz, ..., 0] = torch.from_numpy(G.real.astype(f32))
            t[kz0:kz0 + nkz, ..., 1] = torch.from_numpy(G.imag.astype(f32))

    def c2r(self, x0, nx):
        N = self.N
        for a in range(3):
            t = self.spec[1 + a][:, x0:x0 + nx].numpy()
            c = np.transpose(t[..., 0] + 1j * t[..., 1].astype(np.float64), (1, 2, 0))
            self.meshes[a][x0:x0 + nx] = np.fft.irfft(c, n=N, axis=2) * N

    def _gather(self, pos, x0, nx):
        N = self.N
        out = np.zeros((3, len(pos)), dtype=f32)
        if len(pos) == 0:
            return out
        iI, I1, J, J1, K, K1, D1, D2, D3, T1, T2, T3 = R._cic_index(pos, N, self.L)
        for a in range(3):
            m = self.meshes[a].astype(f32)
            f = np.zeros(len(pos), dtype=f32)
            for ix, wx in ((iI, T1), (I1, D1)):
                ok = (ix >= x0) & (ix < x0 + nx)
                i = np.where(ok, ix, x0)

                def term(jy, kz, wa, wc):
                    return (((m[i, jy, kz] * wa).astype(f32) * wx).astype(f32) * wc).astype(f32)
                g = (((term(J, K, T3, T2) + term(J, K1, D3, T2)).astype(f32)
                      + term(J1, K, T3, D2)).astype(f32) + term(J1, K1, D3, D2)).astype(f32)
                f = np.where(ok, (f + g).astype(f32), f)
            out[a] = f
        return out

    def interp(self, x0, nx, bx, bf):
        self.f[:] = torch.from_numpy(self._gather(self.rows[:, :3].numpy(), x0, nx))
        if bx.shape[1]:
            bf[:] = torch.from_numpy(self._gather(bx.T.numpy(), x0, nx))
