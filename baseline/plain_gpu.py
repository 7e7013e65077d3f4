"""Plain per-op PyTorch-GPU batched LM-IK — the comparison path for the fused kernel.

The reference's ``solve_ik`` is single-instance (``src/better_robot/tasks/ik.py:150-266``);
this is the same method written the way the reference writes it — one torch op
per SE3 operation, per joint, per residual (``kinematics/forward.py:110-129``,
``kinematics/jacobian.py:172-227``, ``residuals/pose.py:58-103``,
``lie/tangents.py:184-207``, ``optim/optimizers/levenberg_marquardt.py:83-131``) —
batched over problems with a per-problem damping and accept mask.  No fusion,
no CUDA graphs, no custom kernels: every op is a stock torch launch.  Problems
with fewer targets than the batch maximum carry zero-weight target rows, which
contribute nothing to r, J, J^T J or J^T r.

Used only by ``bench.py`` to measure the "plain GPU" arm.
"""

from __future__ import annotations

import math

import torch


def _quat_mul(a, b):
    ax, ay, az, aw = a.unbind(-1)
    bx, by, bz, bw = b.unbind(-1)
    return torch.stack([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                        aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz], -1)


def _act(q, p):
    u, w = q[..., :3], q[..., 3:4]
    u, p = torch.broadcast_tensors(u, p)
    c1 = torch.linalg.cross(u, p, dim=-1) + w * p
    return p + 2.0 * torch.linalg.cross(u, c1, dim=-1)


def _compose(a, b):
    return torch.cat([a[..., :3] + _act(a[..., 3:7], b[..., :3]), _quat_mul(a[..., 3:7], b[..., 3:7])], -1)


def _inverse(T):
    qi = T[..., 3:7] * T.new_tensor([-1.0, -1.0, -1.0, 1.0])
    return torch.cat([-_act(qi, T[..., :3]), qi], -1)


def _hat(v):
    z = torch.zeros_like(v[..., 0])
    return torch.stack([torch.stack([z, -v[..., 2], v[..., 1]], -1), torch.stack([v[..., 2], z, -v[..., 0]], -1),
                        torch.stack([-v[..., 1], v[..., 0], z], -1)], -2)


def _quat_to_matrix(q):
    x, y, z, w = q.unbind(-1)
    return torch.stack([torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                        torch.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                        torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], -2)


def _so3_log(q):
    q = torch.where(q[..., 3:4] < 0, -q, q)
    u, w = q[..., :3], q[..., 3:4]
    s2 = (u * u).sum(-1, keepdim=True)
    s = s2.clamp(min=0).sqrt()
    th = 2.0 * torch.atan2(s, w.clamp(-1.0, 1.0))
    f = torch.where(s2 < 0.25e-8, 2.0 + s2 * (2.0 / 3.0), th / s.clamp(min=1e-30))
    return f * u


def _se3_log(T):
    w = _so3_log(T[..., 3:7])
    th2 = (w * w).sum(-1, keepdim=True)
    th = th2.clamp(min=0).sqrt()
    cot = torch.cos(th / 2) / torch.sin(th / 2).clamp(min=1e-30)
    c = torch.where(th2 < 1e-8, 1.0 / 12.0 + th2 / 720.0, 1.0 / th2.clamp(min=1e-30) - cot / (2 * th.clamp(min=1e-30)))
    W = _hat(w)
    Vi = torch.eye(3, device=T.device, dtype=T.dtype) - 0.5 * W + c[..., None] * (W @ W)
    return torch.cat([(Vi @ T[..., :3, None])[..., 0], w], -1)


def _se3_exp(xi):
    v, w = xi[..., :3], xi[..., 3:]
    th2 = (w * w).sum(-1, keepdim=True)
    th = th2.clamp(min=0).sqrt()
    small = th2 < 1e-8
    b = torch.where(small, 0.5 - th2 / 24.0, (1.0 - torch.cos(th)) / th2.clamp(min=1e-30))
    c = torch.where(small, 1.0 / 6.0 - th2 / 120.0, (th - torch.sin(th)) / (th * th2).clamp(min=1e-30))
    W = _hat(w)
    V = torch.eye(3, device=xi.device, dtype=xi.dtype) + b[..., None] * W + c[..., None] * (W @ W)
    k = torch.where(small, 0.5 - th2 / 48.0, torch.sin(th / 2) / th.clamp(min=1e-30))
    return torch.cat([(V @ v[..., None])[..., 0], k * w, torch.cos(th / 2)], -1)


def _jr_inv(xi):
    V, W = _hat(xi[..., :3]), _hat(xi[..., 3:])
    Z = torch.zeros_like(W)
    ad = torch.cat([torch.cat([W, V], -1), torch.cat([Z, W], -1)], -2)
    I6 = torch.eye(6, device=xi.device, dtype=xi.dtype).expand_as(ad)
    res, pw = I6.clone(), I6.clone()
    for k in range(1, 10):
        pw = pw @ ad
        res = res + ((-1.0) ** k) / math.factorial(k + 1) * pw
    return torch.linalg.inv(res)


class PlainLM:
    """Batched per-op LM for one robot class (model tables taken from the Model)."""

    def __init__(self, model, device):
        self.m = model
        self.dev = device
        self.P = model.joint_placements.to(device=device, dtype=torch.float32)
        self.kinds = [jm.kind for jm in model.joint_models]
        ax = {"revolute_rx": (1, 0, 0), "revolute_ry": (0, 1, 0), "revolute_rz": (0, 0, 1)}
        self.axes = [torch.tensor(ax.get(k, (0, 0, 1)), dtype=torch.float32, device=device) for k in self.kinds]
        self.lo = model.lower_pos_limit.to(device=device, dtype=torch.float32)
        self.hi = model.upper_pos_limit.to(device=device, dtype=torch.float32)
        nq, nv = model.nq, model.nv
        self.dq_dv = torch.zeros(nq, nv, device=device)
        for j, k in enumerate(self.kinds):
            if model.nqs[j] == 1 and model.nvs[j] == 1:
                self.dq_dv[model.idx_qs[j], model.idx_vs[j]] = 1.0

    def fk(self, q):
        m = self.m
        world = [None] * m.njoints
        ident = q.new_tensor([0, 0, 0, 0, 0, 0, 1.0]).expand(q.shape[0], 7)
        for j in m.topo_order:
            k = self.kinds[j]
            if k.startswith("revolute"):
                half = q[:, m.idx_qs[j]] / 2
                Tj = torch.cat([torch.zeros(q.shape[0], 3, device=q.device),
                                torch.sin(half)[:, None] * self.axes[j], torch.cos(half)[:, None]], -1)
            elif k == "free_flyer":
                qj = q[:, m.idx_qs[j]:m.idx_qs[j] + 7]
                Tj = torch.cat([qj[:, :3], qj[:, 3:] / qj[:, 3:].norm(dim=-1, keepdim=True).clamp(min=1e-8)], -1)
            else:
                Tj = ident
            loc = _compose(self.P[j].expand(q.shape[0], 7), Tj)
            p = m.parents[j]
            world[j] = loc if p < 0 else _compose(world[p], loc)
        return world

    def frame_pose(self, world, f):
        fr = self.m.frames[f]
        return _compose(world[fr.parent_joint], fr.joint_placement.to(self.dev, torch.float32).expand(
            world[0].shape[0], 7))

    def frame_jac_lwa(self, world, f):
        m = self.m
        fr = self.m.frames[f]
        B = world[0].shape[0]
        J = torch.zeros(B, 6, m.nv, device=self.dev)
        for j in m.supports[fr.parent_joint]:
            nvj = m.nvs[j]
            if nvj == 0:
                continue
            T = world[j]
            R = _quat_to_matrix(T[:, 3:7])
            if self.kinds[j] == "free_flyer":
                S = torch.eye(6, device=self.dev).expand(B, 6, 6)
            else:
                S = torch.zeros(B, 6, 1, device=self.dev)
                S[:, 3:, 0] = self.axes[j]
            RSa = R @ S[:, 3:]
            v = m.idx_vs[j]
            J[:, :3, v:v + nvj] = R @ S[:, :3] + _hat(T[:, :3]) @ RSa
            J[:, 3:, v:v + nvj] = RSa
        Tf = self.frame_pose(world, f)
        lin = J[:, :3] - _hat(Tf[:, :3]) @ J[:, 3:]
        return torch.cat([lin, J[:, 3:]], -2), Tf

    def residual_jacobian(self, q, frame_ids, targets, tmask, q_rest, w, want_jac=True):
        """Stacked r (B, dim) and J (B, dim, nv); targets (B, K, 7), tmask (B, K) 0/1 weights."""
        world = self.fk(q)
        wp, wo, wl, wr = w
        wvec = q.new_tensor([wp] * 3 + [wo] * 3)
        rs, Js = [], []
        for i, f in enumerate(frame_ids):
            if want_jac:
                Jlwa, Tee = self.frame_jac_lwa(world, f)
            else:
                Tee = self.frame_pose(world, f)
            xi = _se3_log(_compose(_inverse(targets[:, i]), Tee))
            mk = tmask[:, i:i + 1]
            rs.append(xi * wvec * mk)
            if want_jac:
                RT = _quat_to_matrix(Tee[:, 3:7]).mT
                Jl = torch.cat([RT @ Jlwa[:, :3], RT @ Jlwa[:, 3:]], -2)
                Js.append((_jr_inv(xi) @ Jl) * wvec[:, None] * mk[..., None])
        rl = torch.cat([torch.clamp(self.lo - q, min=0.0), torch.clamp(q - self.hi, min=0.0)], -1)
        rs.append(torch.nan_to_num(rl, nan=0.0, posinf=0.0, neginf=0.0) * wl)
        m = self.m
        d = []
        for j, k in enumerate(self.kinds):
            if m.nqs[j] == 0:
                continue
            iq = m.idx_qs[j]
            if k == "free_flyer":
                d.append(_se3_log(_compose(_inverse(q_rest[:, iq:iq + 7]), q[:, iq:iq + 7])))
            else:
                d.append(q[:, iq:iq + 1] - q_rest[:, iq:iq + 1])
        rs.append(torch.cat(d, -1) * wr)
        r = torch.cat(rs, -1)
        if not want_jac:
            return r, None
        ld = torch.where(q < self.lo, -1.0, 0.0)
        ud = torch.where(q > self.hi, 1.0, 0.0)
        Js.append(torch.cat([ld[..., None] * self.dq_dv, ud[..., None] * self.dq_dv], -2) * wl)
        Js.append(torch.eye(m.nv, device=self.dev).expand(q.shape[0], m.nv, m.nv) * wr)
        return r, torch.cat(Js, -2)

    def integrate(self, q, dv):
        m = self.m
        parts = []
        for j, k in enumerate(self.kinds):
            if m.nqs[j] == 0:
                continue
            iq, iv = m.idx_qs[j], m.idx_vs[j]
            if k == "free_flyer":
                n = _compose(q[:, iq:iq + 7], _se3_exp(dv[:, iv:iv + 6]))
                parts.append(torch.cat([n[:, :3], n[:, 3:] / n[:, 3:].norm(dim=-1, keepdim=True).clamp(min=1e-8)], -1))
            else:
                parts.append(q[:, iq:iq + 1] + dv[:, iv:iv + 1])
        return torch.cat(parts, -1)

    def solve(self, frame_ids, targets, tmask, q0, q_rest, *, weights=(1.0, 1.0, 0.1, 1e-3), lam0=1e-3,
              factor=10.0, tol=1e-6, max_iter=100):
        q = q0.clone()
        B = q.shape[0]
        r, _ = self.residual_jacobian(q, frame_ids, targets, tmask, q_rest, weights, want_jac=False)
        cost = 0.5 * (r * r).sum(-1)
        lam = torch.full((B,), lam0, device=self.dev)
        active = torch.ones(B, dtype=torch.bool, device=self.dev)
        conv = torch.zeros(B, dtype=torch.bool, device=self.dev)
        iters = torch.full((B,), max_iter, dtype=torch.int32, device=self.dev)
        eye = torch.eye(self.m.nv, device=self.dev)
        for it in range(max_iter):
            r_cur, J = self.residual_jacobian(q, frame_ids, targets, tmask, q_rest, weights)
            JtJ = J.mT @ J
            Jtr = (J.mT @ r_cur[..., None])[..., 0]
            H = JtJ + lam[:, None, None] * eye
            L, info = torch.linalg.cholesky_ex(H)
            dv = torch.cholesky_solve(-Jtr[..., None], L)[..., 0]
            bad = info != 0
            if bool(bad.any()):  # Cholesky.solve falls back to lstsq (optim/solvers/cholesky.py:16-20)
                dv = torch.where(bad[:, None], torch.linalg.lstsq(H, -Jtr[..., None]).solution[..., 0], dv)
            qn = torch.minimum(torch.maximum(self.integrate(q, dv), self.lo), self.hi)
            rn, _ = self.residual_jacobian(qn, frame_ids, targets, tmask, q_rest, weights, want_jac=False)
            cn = 0.5 * (rn * rn).sum(-1)
            acc = (cn < cost) & active
            q = torch.where(acc[:, None], qn, q)
            cost = torch.where(acc, cn, cost)
            lam = torch.where(acc, (lam / factor).clamp(min=1e-10),
                              torch.where(active, (lam * factor).clamp(max=1e8), lam))
            done = acc & (Jtr.norm(dim=-1) < tol)
            iters = torch.where(done, torch.full_like(iters, it + 1), iters)
            conv = conv | done
            active = active & ~done
            if it % 10 == 9 and not bool(active.any()):
                break
        return q, conv, iters
