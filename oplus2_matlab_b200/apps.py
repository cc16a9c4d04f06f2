"""The reference apps' main programs, restated over the OP2 API.

Airfoil follows airfoil/airfoil_op.cpp:112-303 and Jac follows
jac1/jac_op.cpp / jac2/jac_op.cpp: the same sets, maps, datasets, constants
and op_par_loop calls, in the same order.  Tests and the benchmark drive the
library through these, exactly as the generated C mains would.
"""
import math

import numpy as np

from . import api
from .api import (OP_INC, OP_MAX, OP_READ, OP_RW, OP_WRITE, op_arg_dat, op_arg_gbl,
                  op_decl_const, op_decl_dat, op_decl_map, op_decl_set)


def airfoil_consts(dtype):
    """gam, gm1, cfl, eps, mach, alpha, qinf[4] as airfoil/airfoil.cpp:175-199
    computes them.  The FP64 form is the reference's mechanical float->double
    variant, whose literals stay float (1.4f, 0.9f, ...)."""
    if np.dtype(dtype) == np.float32:
        f = np.float32
        gam = f(1.4)
        gm1 = f(gam - f(1.0))
        cfl, eps, mach = f(0.9), f(0.05), f(0.4)
        alpha = f(f(3.0) * np.arctan(f(1.0)) / f(45.0))
        p = r = f(1.0)
        u = f(np.sqrt(f(gam * p / r)) * mach)
        e = f(p / (r * gm1) + f(f(0.5) * u) * u)
        qinf = np.array([r, r * u, 0.0, r * e], np.float32)
        return dict(gam=gam, gm1=gm1, cfl=cfl, eps=eps, mach=mach, alpha=alpha, qinf=qinf)
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    gam = f32(1.4)
    gm1 = gam - 1.0
    cfl, eps, mach = f32(0.9), f32(0.05), f32(0.4)
    alpha = float(np.float32(np.float32(3.0) * np.arctan(np.float32(1.0)) / np.float32(45.0)))
    p = r = 1.0
    u = math.sqrt(gam * p / r) * mach
    e = p / (r * gm1) + 0.5 * u * u
    qinf = np.array([r, r * u, 0.0, r * e], np.float64)
    return dict(gam=gam, gm1=gm1, cfl=cfl, eps=eps, mach=mach, alpha=alpha, qinf=qinf)


class Airfoil:
    """airfoil_op.cpp with the library: declare, then iterate()."""

    def __init__(self, mesh, dtype=np.float32, consts=None, q0=None, state=None):
        self.dtype = t = np.dtype(dtype)
        tn = "float" if t == np.float32 else "double"
        self.tn = tn
        self.mesh = mesh
        K = consts or airfoil_consts(t)
        self.K = K
        nc = mesh.ncell
        # flow field initialised to free stream, residual to zero (airfoil.cpp:193-199)
        self.q = np.tile(np.asarray(K["qinf"], t), (nc, 1)) if q0 is None else np.array(q0, t)
        self.qold = np.zeros((nc, 4), t)
        self.res = np.zeros((nc, 4), t)
        self.adt = np.zeros((nc, 1), t)
        if state is not None:  # start from a given flow state instead
            for k in ("q", "qold", "res", "adt"):
                getattr(self, k)[...] = np.asarray(state[k], t).reshape(getattr(self, k).shape)
        self.x = np.ascontiguousarray(mesh.x(t))
        self.bound = np.ascontiguousarray(mesh.bound.reshape(-1, 1))

        self.nodes = op_decl_set(mesh.nnode, "nodes")
        self.edges = op_decl_set(mesh.nedge, "edges")
        self.bedges = op_decl_set(mesh.nbedge, "bedges")
        self.cells = op_decl_set(mesh.ncell, "cells")
        self.pedge = op_decl_map(self.edges, self.nodes, 2, mesh.edge, "pedge")
        self.pecell = op_decl_map(self.edges, self.cells, 2, mesh.ecell, "pecell")
        self.pbedge = op_decl_map(self.bedges, self.nodes, 2, mesh.bedge, "pbedge")
        self.pbecell = op_decl_map(self.bedges, self.cells, 1, mesh.becell, "pbecell")
        self.pcell = op_decl_map(self.cells, self.nodes, 4, mesh.cell, "pcell")
        self.p_bound = op_decl_dat(self.bedges, 1, "int", self.bound, "p_bound")
        self.p_x = op_decl_dat(self.nodes, 2, tn, self.x, "p_x")
        self.p_q = op_decl_dat(self.cells, 4, tn, self.q, "p_q")
        self.p_qold = op_decl_dat(self.cells, 4, tn, self.qold, "p_qold")
        self.p_adt = op_decl_dat(self.cells, 1, tn, self.adt, "p_adt")
        self.p_res = op_decl_dat(self.cells, 4, tn, self.res, "p_res")
        for name in ("gam", "gm1", "cfl", "eps", "mach", "alpha"):
            op_decl_const(name, 1, tn, K[name])
        op_decl_const("qinf", 4, tn, K["qinf"])

        self.rms = np.zeros(1, t)
        pX, pQ, pQo, pA, pR = self.p_x, self.p_q, self.p_qold, self.p_adt, self.p_res
        self.loops = {
            "save_soln": (self.cells, [op_arg_dat(pQ, -1, None, 4, tn, OP_READ),
                                       op_arg_dat(pQo, -1, None, 4, tn, OP_WRITE)]),
            "adt_calc": (self.cells, [op_arg_dat(pX, 0, self.pcell, 2, tn, OP_READ),
                                      op_arg_dat(pX, 1, self.pcell, 2, tn, OP_READ),
                                      op_arg_dat(pX, 2, self.pcell, 2, tn, OP_READ),
                                      op_arg_dat(pX, 3, self.pcell, 2, tn, OP_READ),
                                      op_arg_dat(pQ, -1, None, 4, tn, OP_READ),
                                      op_arg_dat(pA, -1, None, 1, tn, OP_WRITE)]),
            "res_calc": (self.edges, [op_arg_dat(pX, 0, self.pedge, 2, tn, OP_READ),
                                      op_arg_dat(pX, 1, self.pedge, 2, tn, OP_READ),
                                      op_arg_dat(pQ, 0, self.pecell, 4, tn, OP_READ),
                                      op_arg_dat(pQ, 1, self.pecell, 4, tn, OP_READ),
                                      op_arg_dat(pA, 0, self.pecell, 1, tn, OP_READ),
                                      op_arg_dat(pA, 1, self.pecell, 1, tn, OP_READ),
                                      op_arg_dat(pR, 0, self.pecell, 4, tn, OP_INC),
                                      op_arg_dat(pR, 1, self.pecell, 4, tn, OP_INC)]),
            "bres_calc": (self.bedges, [op_arg_dat(pX, 0, self.pbedge, 2, tn, OP_READ),
                                        op_arg_dat(pX, 1, self.pbedge, 2, tn, OP_READ),
                                        op_arg_dat(pQ, 0, self.pbecell, 4, tn, OP_READ),
                                        op_arg_dat(pA, 0, self.pbecell, 1, tn, OP_READ),
                                        op_arg_dat(pR, 0, self.pbecell, 4, tn, OP_INC),
                                        op_arg_dat(self.p_bound, -1, None, 1, "int", OP_READ)]),
            "update": (self.cells, [op_arg_dat(pQo, -1, None, 4, tn, OP_READ),
                                    op_arg_dat(pQ, -1, None, 4, tn, OP_WRITE),
                                    op_arg_dat(pR, -1, None, 4, tn, OP_RW),
                                    op_arg_dat(pA, -1, None, 1, tn, OP_READ),
                                    op_arg_gbl(self.rms, 1, tn, OP_INC)]),
        }
        lib = api.lib()
        self._calls = {}
        for name, (s, args) in self.loops.items():
            arr = (api.op_arg * len(args))(*args)
            self._calls[name] = (api._b(name), s, len(args), arr)
        self._par_loop = lib.op2b_par_loop

    def loop(self, name):
        nm, s, n, arr = self._calls[name]
        self._par_loop(nm, s, n, arr)

    def iteration(self):
        """One outer iteration of airfoil_op.cpp:241-301; returns the printed rms."""
        self.loop("save_soln")
        for _ in range(2):
            self.loop("adt_calc")
            self.loop("res_calc")
            self.loop("bres_calc")
            self.rms[0] = 0
            self.loop("update")
        return self.dtype.type(np.sqrt(self.rms[0] / self.dtype.type(self.mesh.ncell)))

    def iterate(self, niter):
        return np.array([self.iteration() for _ in range(niter)], self.dtype)

    def fetch(self):
        for d in (self.p_q, self.p_qold, self.p_res, self.p_adt):
            api.op_fetch_data(d)
        return dict(q=self.q, qold=self.qold, res=self.res, adt=self.adt)


class Jac:
    """jac1/jac_op.cpp (variant 1) or jac2/jac_op.cpp (variant 2)."""

    def __init__(self, mesh, variant=1):
        self.variant = variant
        self.mesh = mesh
        nn = mesh.nnode
        if variant == 1:
            self.u, self.du = np.zeros(nn, np.float32), np.zeros(nn, np.float32)
            self.A, self.r = mesh.A.reshape(-1, 1).copy(), mesh.r.reshape(-1, 1).copy()
            self.u, self.du = self.u.reshape(-1, 1), self.du.reshape(-1, 1)
            da, du, dd, dr, at = 1, 1, 1, 1, "float"
        else:
            self.u, self.du = np.zeros((nn, 2), np.float32), np.zeros((nn, 3), np.float32)
            self.A, self.r = mesh.A.copy(), mesh.r.copy()
            da, du, dd, dr, at = 3, 2, 3, 2, "double"
        self.nodes = op_decl_set(nn, "nodes")
        self.edges = op_decl_set(mesh.nedge, "edges")
        self.ppedge = op_decl_map(self.edges, self.nodes, 2, mesh.pp, "ppedge")
        self.p_A = op_decl_dat(self.edges, da, at, self.A, "p_A")
        self.p_r = op_decl_dat(self.nodes, dr, "float", self.r, "p_r")
        self.p_u = op_decl_dat(self.nodes, du, "float", self.u, "p_u")
        self.p_du = op_decl_dat(self.nodes, dd, "float", self.du, "p_du")
        # jac2/jac.cpp:137-140 declares alpha twice; the second value holds
        if variant == 2:
            op_decl_const("alpha", 1, "float", 2.0)
        op_decl_const("alpha", 1, "float", 1.0)
        self.beta = np.ones(1, np.float32)
        self.u_sum = np.zeros(1, np.float32)
        self.u_max = np.zeros(1, np.float32)
        self.res_args = [op_arg_dat(self.p_A, -1, None, da, at, OP_READ),
                         op_arg_dat(self.p_u, 1, self.ppedge, du, "float", OP_READ),
                         op_arg_dat(self.p_du, 0, self.ppedge, dd, "float", OP_INC),
                         op_arg_gbl(self.beta, 1, "float", OP_READ)]
        self.upd_args = [op_arg_dat(self.p_r, -1, None, dr, "float", OP_READ),
                         op_arg_dat(self.p_du, -1, None, dd, "float", OP_RW),
                         op_arg_dat(self.p_u, -1, None, du, "float", OP_INC),
                         op_arg_gbl(self.u_sum, 1, "float", OP_INC),
                         op_arg_gbl(self.u_max, 1, "float", OP_MAX)]

    def iteration(self):
        """One iteration of jac1/jac_op.cpp:166-183; returns (u_max, u_sum)."""
        api.op_par_loop("res", self.edges, *self.res_args)
        self.u_sum[0] = 0
        self.u_max[0] = 0
        api.op_par_loop("update", self.nodes, *self.upd_args)
        return float(self.u_max[0]), float(self.u_sum[0])

    def iterate(self, niter):
        return [self.iteration() for _ in range(niter)]

    def fetch(self):
        api.op_fetch_data(self.p_u)
        return self.u
