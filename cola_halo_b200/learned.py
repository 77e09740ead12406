"""Learned small-scale force correction on a coarse mesh (cg_net_* in
colagpu.h): training on PM-generated pairs and learned-correction runs."""
import ctypes

import numpy as np

from . import _lib
from .schedule import output_scale_factors, run_time_loop


class ConvNet:
    def __init__(self, ngrid, seed=1):
        self.lib = _lib.load()
        self.ngrid = ngrid
        h = ctypes.c_void_p()
        _lib.check(self.lib.cg_net_create(ctypes.byref(h), ngrid, seed), "cg_net_create")
        self.h = h
        self.nparams = self.lib.cg_net_num_params()

    def close(self):
        if self.h:
            self.lib.cg_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        _lib.check(self.lib.cg_net_get_params(self.h, p.ctypes.data), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(self.lib.cg_net_set_params(self.h, p.ctypes.data), "set_params")

    def set_scales(self, in_delta, in_phi, out_scale):
        _lib.check(self.lib.cg_net_set_scales(self.h, in_delta, in_phi, out_scale), "scales")

    def tensor_cores(self, on):
        _lib.check(self.lib.cg_net_set_tensor_cores(self.h, 1 if on else 0), "tensor cores")

    def forward_host(self, in2):
        n = self.ngrid
        a = np.ascontiguousarray(in2, dtype=np.float32)
        out = np.zeros((n, n, n, 3), dtype=np.float32)
        _lib.check(self.lib.cg_net_forward_host(self.h, a.ctypes.data, out.ctypes.data),
                   "forward_host")
        return out

    def backward_host(self, in2, grad3):
        a = np.ascontiguousarray(in2, dtype=np.float32)
        g = np.ascontiguousarray(grad3, dtype=np.float32)
        out = np.zeros(self.nparams, dtype=np.float32)
        _lib.check(self.lib.cg_net_backward_host(self.h, a.ctypes.data, g.ctypes.data,
                                                 out.ctypes.data), "backward_host")
        return out

    def train_step(self, coarse, fine, lr):
        loss = ctypes.c_double()
        _lib.check(self.lib.cg_net_train_step(self.h, coarse.h, fine.h, lr, ctypes.byref(loss)),
                   "cg_net_train_step")
        return loss.value

    def forces(self, coarse):
        _lib.check(self.lib.cg_net_forces(self.h, coarse.h), "cg_net_forces")

    def run(self, coarse, sched, zout=(0.0,)):
        """The reference time loop on the coarse realization with corrected
        forces; returns the snapshots."""
        snaps = []
        run_time_loop(sched, output_scale_factors(zout), move=coarse.move,
                      force=lambda: self.forces(coarse), kick=coarse.kick, drift=coarse.drift,
                      snapshot=lambda a, i: snaps.append((a, coarse.snapshot(a))))
        return snaps


def copy_particles(dst, src):
    _lib.check(_lib.load().cg_sim_copy_particles(dst.h, src.h), "cg_sim_copy_particles")
