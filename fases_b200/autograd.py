"""torch.autograd front end of the solver's discrete adjoint.

`impulse_responses` and `misfit` are differentiable functions of torch tensors holding the ADE
material coefficients, the source strengths, the cPML profile parameters and the initial
pressure field. Their backward passes run fz_misfit_gradient_ex: a forward pass with checkpoints,
recomputation of each segment and the reverse sweep of the stepping kernels' adjoint. The
reference has no differentiable solver; it fits materials in the frequency domain
(common/fminconFIT.py:239-348, common/vectFIT.py:335-459).

    room = Room(S, oid, prm, rec_cells=..., src_cells=..., u_s=..., nsteps=800, K=2, L=2)
    theta = torch.tensor(room.materials0, requires_grad=True)      # [nMat, 1 + 2K + 4L]
    ir = impulse_responses(room, theta)                           # [n_rec, nsteps], float64
    loss = ((ir - target) ** 2).sum(); loss.backward()            # theta.grad

Material rows use the gradient layout of fz_misfit_gradient: Rinf, A[K], zeta[K], B[L], C[L],
alpha[L], beta[L].
"""
import numpy as np
import torch

from .solver import Solver, params as make_params


def unpack_materials(rows, K, L):
    """[nMat, 1 + 2K + 4L] rows -> (Rinf, A, zeta, B, C, alpha, beta) for Solver.set_materials."""
    m = np.asarray(rows, dtype=np.float64).reshape(-1, 1 + 2 * K + 4 * L)
    o = 1 + 2 * K
    return (m[:, 0], m[:, 1:1 + K], m[:, 1 + K:o], m[:, o:o + L], m[:, o + L:o + 2 * L], m[:, o + 2 * L:o + 3 * L],
            m[:, o + 3 * L:o + 4 * L])


def pack_materials(Rinf, A, zeta, B, C, alpha, beta):
    """Inverse of unpack_materials."""
    Rinf = np.asarray(Rinf, dtype=np.float64).reshape(-1, 1)
    n = Rinf.shape[0]
    parts = [np.asarray(x, dtype=np.float64).reshape(n, -1) for x in (A, zeta, B, C, alpha, beta)]
    return np.concatenate([Rinf] + parts, axis=1)


class Room:
    """The fixed part of a differentiable solve: grid, geometry, receivers, source cells and
    waveform, step count. `solver(...)` builds a Solver at step 0 from the differentiable values.

    S, oid: the geometry arrays of Solver.load_geometry; prm: solver parameters (fz_params, or a
    dict for solver.params); materials0: [nMat, 1 + 2K + 4L] default material rows; sval0: default
    source strengths; p0: default initial pressure ([Nz, Ny, Nx]) or None."""

    def __init__(self, S, oid, prm, rec_cells, nsteps, materials0, src_cells=(), sval0=(), src_opt=0, u_s=None,
                 freq=None, p0=None, K=1, L=1, segment_steps=250):
        self.S = np.ascontiguousarray(S, dtype=np.float32)
        self.oid = np.ascontiguousarray(oid, dtype=np.uint8)
        self.prm = prm
        self.rec_cells = np.asarray(rec_cells, dtype=np.int32).reshape(-1, 3)
        self.nsteps = int(nsteps)
        self.K, self.L = int(K), int(L)
        self.materials0 = np.asarray(materials0, dtype=np.float64).reshape(-1, 1 + 2 * self.K + 4 * self.L)
        self.src_cells = np.asarray(src_cells, dtype=np.int32).reshape(-1, 3)
        self.sval0 = np.asarray(sval0, dtype=np.float64).reshape(-1)
        self.src_opt = int(src_opt)
        self.u_s = None if u_s is None else np.asarray(u_s, dtype=np.float64)
        self.freq = None if freq is None else np.asarray(freq, dtype=np.float64)
        self.p0 = None if p0 is None else np.asarray(p0, dtype=np.float64)
        self.segment_steps = int(segment_steps)

    def _params(self, pml):
        if isinstance(self.prm, dict):
            kw = dict(self.prm)
        else:
            p = self.prm
            kw = dict(h=p.h, c=p.c, rho=p.rho, dt=p.dt, pml=tuple(p.pml), pml_cells=p.pml_cells,
                      precision="fp64" if p.precision == 1 else "fp32", device=p.device, tol_cells=p.tol_cells,
                      pml_R0=p.pml_R0, pml_kappa_max=p.pml_kappa_max, pml_alpha_max=p.pml_alpha_max,
                      pml_order=p.pml_order)
        if pml is not None:
            kw["pml_R0"], kw["pml_kappa_max"], kw["pml_alpha_max"] = (float(x) for x in pml)
        return make_params(**kw)

    def solver(self, materials=None, sval=None, pml=None, p0=None):
        s = Solver(self._params(pml))
        s.load_geometry(self.S, self.oid)
        s.set_materials(*unpack_materials(self.materials0 if materials is None else materials, self.K, self.L))
        if self.src_cells.shape[0] > 0:
            s.set_sources(self.src_cells, self.sval0 if sval is None else sval, src_opt=self.src_opt, u_s=self.u_s,
                          freq=self.freq)
        s.set_receivers(self.rec_cells, self.nsteps)
        p0 = self.p0 if p0 is None else p0
        if p0 is not None:
            s.set_fields(p=p0)
        return s


def _np(t):
    return None if t is None else t.detach().to("cpu", torch.float64).numpy()


def _grads(g, like, req):
    """Gradients in the order (materials, sval, pml, p0), as tensors shaped and placed like the
    inputs (None where the input needs none)."""
    out = []
    for t, r, key in zip(like, req, ("raw", "sval", "pml", "initial")):
        if t is None or not r:
            out.append(None)
            continue
        v = g[key]
        if key == "pml":
            v = np.array([v["R0"], v["kappa_max"], v["alpha_max"]])
        elif key == "initial":
            v = v[0]
        out.append(torch.as_tensor(np.asarray(v).reshape(t.shape), dtype=t.dtype, device=t.device))
    return out


def _run_gradient(room, values, req, target, cotangent):
    s = room.solver(*values)
    try:
        return s.misfit_gradient(target, nsteps=room.nsteps, segment_steps=room.segment_steps, sources=req[1],
                                 pml=req[2], initial=req[3], cotangent=cotangent)
    finally:
        s.close()


def _req(like):
    return tuple(t is not None and t.requires_grad for t in like)


class _ImpulseResponses(torch.autograd.Function):
    @staticmethod
    def forward(ctx, room, materials, sval, pml, p0):
        like = (materials, sval, pml, p0)
        values = tuple(_np(t) for t in like)
        s = room.solver(*values)
        try:
            s.run(room.nsteps)
            ir = s.ir()[:, :room.nsteps].copy()
        finally:
            s.close()
        ctx.room, ctx.values, ctx.req = room, values, _req(like)
        ctx.like = tuple(None if t is None else t.detach() for t in like)
        return torch.as_tensor(ir, device=materials.device)

    @staticmethod
    def backward(ctx, g_ir):
        g = _run_gradient(ctx.room, ctx.values, ctx.req, np.ascontiguousarray(_np(g_ir)), cotangent=True)
        return (None,) + tuple(_grads(g, ctx.like, ctx.req))


class _Misfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, room, target, materials, sval, pml, p0):
        like = (materials, sval, pml, p0)
        values = tuple(_np(t) for t in like)
        req = _req(like)
        g = _run_gradient(room, values, req, np.ascontiguousarray(_np(target)), cotangent=False)
        ctx.grads = _grads(g, like, req)
        return torch.tensor(g["J"], dtype=torch.float64, device=materials.device)

    @staticmethod
    def backward(ctx, gJ):
        return (None, None) + tuple(None if x is None else x * gJ.to(x.dtype) for x in ctx.grads)


def impulse_responses(room, materials, sval=None, pml=None, p0=None):
    """Receiver traces [n_rec, nsteps] (float64) of `room` with the given material rows, source
    strengths, cPML parameters (R0, kappa_max, alpha_max) and initial pressure; differentiable in
    each tensor that requires grad. The backward pass costs one forward pass with checkpoints plus
    the reverse sweep (the trajectory is not kept between the passes)."""
    return _ImpulseResponses.apply(room, materials, sval, pml, p0)


def misfit(room, target, materials, sval=None, pml=None, p0=None):
    """J = sum (IR - target)^2 with its gradient computed in the same call (one forward pass with
    checkpoints and one reverse sweep); backward only scales the stored gradient."""
    return _Misfit.apply(room, target, materials, sval, pml, p0)
