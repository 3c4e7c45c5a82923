"""Differentiable multi-step particle-mesh chain on the CUDA kernels.

Per step k (particles ordered by their initial brick and cell, no
rebinning; the gradients come back in the caller's order):
    rho_k   = deposit(x_k, m)                    lf2_pm_deposit      (CIC, projections.hpp:75-184)
    F_k     = stencil27(rho_k, S)                lf2_stencil27       (the grid operator), or
    F_k     = pm_force(rho_k)                    lf2_pm_force4       (the FFT Poisson force)
    G_k     = gather(x_k, F_k)                   lf2_pm_gather       (CIC gather of updateVel)
    v_{k+1} = v_k + dt G_k ;  x_{k+1} = x_k + dt v_{k+1}             lf2_pm_kick_drift
(the last two in one pass, lf2_pm_step)
and finally rho_K = deposit(x_K, m), loss = sum_g w_g rho_K(g).

`PMChain` is a torch.autograd.Function whose backward runs the hand-written
adjoint kernels (lf2_pm_*_adjoint, lf2_stencil27_adjoint,
lf2_pm_force4_adjoint) in reverse.
Particle states are checkpointed every `checkpoint_every` steps and the
states in between are recomputed during the backward pass; the grid fields
rho_k and F_k of every step are kept (4 floats per lattice site per step).
Gradients are returned for the initial positions (box units), velocities,
masses, the 81 stencil weights (stencil operator only) and the loss weights.
The PM operator solves lap7(phi) = coupling (rho - mean rho) by FFT and takes
F = -grad phi by central differences (the operator of lf2_pm_force; cubic
lattices).
"""
import ctypes

import torch

from . import _lib
from .core import Context


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _check(ctx, status, what):
    _lib.check(ctx.h, status, what)


def positions_to_state(pos, n, res):
    """Box-unit positions (float64) -> int32 cell, FP32 in-cell offset."""
    u = pos / res
    fl = torch.floor(u)
    off = (u - fl).to(torch.float32)
    carry = off >= 1.0
    off = torch.where(carry, torch.zeros_like(off), off)
    fl = fl + carry.to(fl.dtype)
    nn = torch.tensor(n, dtype=torch.int64, device=pos.device)
    ci = torch.remainder(fl.to(torch.int64), nn)
    cell = ci[:, 0] + n[0] * (ci[:, 1] + n[1] * ci[:, 2])
    return cell.to(torch.int32).contiguous(), off.contiguous()


class _Ops:
    """The kernel calls of one chain, bound to a Context."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.lib = _lib.load()
        self.ns = ctx.nsites

    bricks = None  # brick_start of the sorted state: deposits run brick-tiled

    def state_pack(self, pos, vel, mass, inv_res):
        """Caller order: the sort keys (brick, then cell in the brick) and one
        32-byte record per particle (cell, offsets, FP32 velocity and mass)."""
        n = pos.shape[0]
        key = torch.empty(n, dtype=torch.int32, device=pos.device)
        rec = torch.empty(n * 8, dtype=torch.int32, device=pos.device)
        _check(self.ctx, self.lib.lf2_pm_state_pack(self.ctx.h, n, _p(pos), _p(vel), _p(mass),
                                                    inv_res, _p(key), _p(rec)), "pm_state_pack")
        return key, rec

    def state_unpack(self, order, rec):
        """cell, offsets, FP32 velocities and masses of the particles `order`."""
        n = order.numel()
        dev = rec.device
        cell = torch.empty(n, dtype=torch.int32, device=dev)
        off = torch.empty(n, 3, dtype=torch.float32, device=dev)
        vel32 = torch.empty(n, 3, dtype=torch.float32, device=dev)
        m32 = torch.empty(n, dtype=torch.float32, device=dev)
        _check(self.ctx, self.lib.lf2_pm_state_unpack(self.ctx.h, n, _p(order), _p(rec), _p(cell),
                                                      _p(off), _p(vel32), _p(m32)),
               "pm_state_unpack")
        return cell, off, vel32, m32

    def brick_start(self, cell):
        """First slot of every brick among cells sorted by the pack's key."""
        bs = torch.empty(self.ctx.nbricks + 1, dtype=torch.int64, device=cell.device)
        _check(self.ctx, self.lib.lf2_pm_brick_start(self.ctx.h, cell.numel(), _p(cell), _p(bs)),
               "pm_brick_start")
        return bs

    def grads_unorder(self, order, g_off, g_v, g_m, inv_res):
        """FP64 gradients in the caller's order: positions (per box unit),
        velocities, masses."""
        n = order.numel()
        dev = g_off.device
        rec = torch.empty(n * 8, dtype=torch.int32, device=dev)
        g_pos = torch.empty(n, 3, dtype=torch.float64, device=dev)
        g_vel = torch.empty(n, 3, dtype=torch.float64, device=dev)
        g_mass = torch.empty(n, dtype=torch.float64, device=dev)
        _check(self.ctx, self.lib.lf2_pm_grads_unorder(self.ctx.h, n, _p(order), _p(g_off), _p(g_v),
                                                       _p(g_m), inv_res, _p(rec), _p(g_pos),
                                                       _p(g_vel), _p(g_mass)), "pm_grads_unorder")
        return g_pos, g_vel, g_mass

    def deposit(self, cell, off, m, rho):
        if self.bricks is not None:
            _check(self.ctx, self.lib.lf2_pm_deposit_bricks(self.ctx.h, cell.numel(), _p(cell),
                                                            _p(off), _p(m), 0.0, _p(self.bricks),
                                                            _p(rho)), "pm_deposit_bricks")
            return
        _check(self.ctx, self.lib.lf2_pm_deposit(self.ctx.h, cell.numel(), _p(cell), _p(off), _p(m),
                                                 0.0, _p(rho)), "pm_deposit")

    def stencil(self, rho, S, F):
        _check(self.ctx, self.lib.lf2_stencil27(self.ctx.h, _p(rho), _p(S), _p(F)), "stencil27")

    def gather(self, cell, off, F, G):
        _check(self.ctx, self.lib.lf2_pm_gather(self.ctx.h, cell.numel(), _p(cell), _p(off), _p(F),
                                                _p(G)), "pm_gather")

    def kick_drift(self, cell, off, vel, G, dt):
        _check(self.ctx, self.lib.lf2_pm_kick_drift(self.ctx.h, cell.numel(), _p(cell), _p(off),
                                                    _p(vel), _p(G), dt, dt), "pm_kick_drift")

    def deposit_adj(self, cell, off, m, g_rho, g_off, g_m):
        _check(self.ctx, self.lib.lf2_pm_deposit_adjoint(self.ctx.h, cell.numel(), _p(cell), _p(off),
                                                         _p(m), 0.0, _p(g_rho), _p(g_off),
                                                         _p(g_m)), "pm_deposit_adjoint")

    def gather_adj(self, cell, off, F, g_G, g_F, g_off):
        _check(self.ctx, self.lib.lf2_pm_gather_adjoint(self.ctx.h, cell.numel(), _p(cell), _p(off),
                                                        _p(F), _p(g_G), _p(g_F), _p(g_off)),
               "pm_gather_adjoint")

    def stencil_adj(self, rho, S, g_F, g_rho, g_S):
        _check(self.ctx, self.lib.lf2_stencil27_adjoint(self.ctx.h, _p(rho), _p(S), _p(g_F),
                                                        _p(g_rho), _p(g_S)), "stencil27_adjoint")

    def pm_force(self, rho, F, coupling):
        _check(self.ctx, self.lib.lf2_pm_force4(self.ctx.h, _p(rho), _p(F), coupling), "pm_force4")

    def pm_force_adj(self, g_F, g_rho, coupling):
        _check(self.ctx, self.lib.lf2_pm_force4_adjoint(self.ctx.h, _p(g_F), _p(g_rho), coupling),
               "pm_force4_adjoint")

    def fields(self, cell, off, m, S, coupling=None):
        """rho and the float4-per-site force: the stencil S, or the PM force
        when `coupling` is given."""
        dev = cell.device
        rho = torch.zeros(self.ns, dtype=torch.float32, device=dev)
        self.deposit(cell, off, m, rho)
        F = torch.empty(4 * self.ns, dtype=torch.float32, device=dev)  # float4 per site
        if coupling is None:
            self.stencil(rho, S, F)
        else:
            self.pm_force(rho, F, coupling)
        return rho, F

    def step(self, cell, off, vel, F, dt):
        """gather, kick and drift in one pass (lf2_pm_step)."""
        _check(self.ctx, self.lib.lf2_pm_step(self.ctx.h, cell.numel(), _p(cell), _p(off), _p(vel),
                                              _p(F), dt, dt), "pm_step")


class PMChain(torch.autograd.Function):
    @staticmethod
    def forward(fctx, pos0, vel0, mass, S, w, lf2ctx, steps, dt, checkpoint_every, coupling):
        ops = _Ops(lf2ctx)
        res = lf2ctx.res
        # the chain runs on the particles ordered by brick and by cell inside
        # it (the deposits sum each brick in a shared tile, and every access
        # is local); the gradients go back to the caller's order at the end of
        # the backward pass.  The permutations move one 32-byte record per
        # particle.
        key, rec = ops.state_pack(pos0.detach().to(torch.float64).contiguous(),
                                  vel0.detach().to(torch.float64).contiguous(),
                                  mass.detach().to(torch.float64).contiguous(), 1.0 / res)
        order = torch.argsort(key)
        del key
        cell, off, vel, m = ops.state_unpack(order, rec)
        del rec
        # a particle that drifts out of its brick later is deposited on its own
        ops.bricks = ops.brick_start(cell)
        S32 = None if S is None else S.detach().to(torch.float32).contiguous()
        w32 = w.detach().to(torch.float32).contiguous().reshape(-1)
        ckpts, rhos, Fs = {}, [], []
        for k in range(steps):
            if k % checkpoint_every == 0:
                ckpts[k] = (cell.clone(), off.clone(), vel.clone())
            rho, F = ops.fields(cell, off, m, S32, coupling)
            rhos.append(rho)
            Fs.append(F)
            ops.step(cell, off, vel, F, dt)
        rhoK = torch.zeros(lf2ctx.nsites, dtype=torch.float32, device=cell.device)
        ops.deposit(cell, off, m, rhoK)
        loss = torch.dot(w32.to(torch.float64), rhoK.to(torch.float64))
        fctx.lf2 = (lf2ctx, steps, dt, checkpoint_every, ckpts, rhos, Fs, coupling)
        fctx.save_for_backward(cell, off, m, S32, w32, rhoK, order)
        fctx.pos_dtype = pos0.dtype
        fctx.vel_dtype = vel0.dtype
        return loss

    @staticmethod
    def backward(fctx, gloss):
        lf2ctx, steps, dt, every, ckpts, rhos, Fs, coupling = fctx.lf2
        cellK, offK, m, S32, w32, rhoK, order = fctx.saved_tensors
        ops = _Ops(lf2ctx)
        dev = cellK.device
        res = lf2ctx.res
        npart = cellK.numel()
        g = float(gloss)
        g_off = torch.zeros(npart, 3, dtype=torch.float32, device=dev)
        g_v = torch.zeros(npart, 3, dtype=torch.float32, device=dev)
        g_m = torch.zeros(npart, dtype=torch.float32, device=dev)
        g_S = torch.zeros(81, dtype=torch.float32, device=dev)
        ops.deposit_adj(cellK, offK, m, (w32 * g).contiguous(), g_off, g_m)
        seg = {}
        for k in range(steps - 1, -1, -1):
            k0 = (k // every) * every
            if k not in seg:
                # replay the segment from its checkpoint (k is its last step:
                # the segments are visited once, last first, so the
                # checkpoint is consumed), keeping each state
                seg = {}
                if k0 not in ckpts:
                    raise RuntimeError("the chain's backward ran already: its checkpoints are "
                                       "consumed (call backward once per forward)")
                c, o, v = ckpts.pop(k0)
                for j in range(k0, k + 1):
                    seg[j] = (c.clone(), o.clone()) if j < k else (c, o)
                    if j < k:
                        ops.step(c, o, v, Fs[j], dt)
            cell_k, off_k = seg[k]
            # drift x_{k+1} = x_k + dt v_{k+1} (cell units: off += dt/res v)
            g_v += (dt / res) * g_off
            # kick v_{k+1} = v_k + dt G_k
            g_G = (dt * g_v).contiguous()
            g_F = torch.zeros(4 * lf2ctx.nsites, dtype=torch.float32, device=dev)
            ops.gather_adj(cell_k, off_k, Fs[k], g_G, g_F, g_off)
            g_rho = torch.zeros(lf2ctx.nsites, dtype=torch.float32, device=dev)
            if coupling is None:
                ops.stencil_adj(rhos[k], S32, g_F, g_rho, g_S)
            else:
                ops.pm_force_adj(g_F, g_rho, coupling)
            ops.deposit_adj(cell_k, off_k, m, g_rho, g_off, g_m)
        g_pos, g_vel, g_mass = ops.grads_unorder(order, g_off, g_v, g_m, 1.0 / res)
        del g_off, g_v, g_m
        g_w = (rhoK * g).to(torch.float64)
        g_S = None if S32 is None else g_S.to(torch.float64)
        return (g_pos.to(fctx.pos_dtype), g_vel.to(fctx.vel_dtype), g_mass, g_S, g_w,
                None, None, None, None, None)


def pm_chain_loss(ctx: Context, pos0, vel0, mass, S, w, steps=8, dt=0.1, checkpoint_every=2,
                  operator="stencil", coupling=1.0):
    """Loss of the multi-step chain; differentiable in pos0, vel0, mass, w and,
    with operator "stencil", the 81 weights S.  operator "pm" uses the FFT
    Poisson force with `coupling` instead (S is then ignored and may be None)."""
    if operator == "stencil":
        if S is None:
            raise ValueError("the stencil operator needs its 81 weights S")
        return PMChain.apply(pos0, vel0, mass, S, w, ctx, steps, dt, checkpoint_every, None)
    if operator == "pm":
        return PMChain.apply(pos0, vel0, mass, None, w, ctx, steps, dt, checkpoint_every,
                             float(coupling))
    raise ValueError(f"unknown grid operator {operator!r} (stencil or pm)")
