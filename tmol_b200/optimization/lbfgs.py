"""Batched L-BFGS with Armijo backtracking, one independent minimisation
per pose.

The algorithm is limited-memory BFGS with an Armijo backtracking line
search (Nocedal & Wright, Numerical Optimization, 2nd ed., Algorithm 3.1),
applied to every pose at once: coordinates are a [P, L] tensor (L = 3 * max
atoms per pose, padding atoms have zero gradient), curvature pairs are
stored as [m, P, L] ring buffers, and every scalar (step length, energy,
convergence flag) is a length-P vector, so one energy + gradient call
serves all poses.  The search direction uses the compact representation of
the inverse Hessian (Byrd, Nocedal & Schnabel, Math. Prog. 63 (1994), with
H0 = gamma I): with a = S^T g, b = Y^T g, R = upper(S^T Y), D = diag(S^T Y),
v = R^-1 a,  H g = gamma g + S R^-T ((D + gamma Y^T Y) v - gamma b) - gamma Y v,
where S^T Y and Y^T Y are kept up to date one row and column per iteration.  It plays
the role of tmol's LBFGS_Armijo (tmol/optimization/lbfgs_armijo.py:196)
for Cartesian minimisation: same defaults (200 iterations, history 128,
convergence when max |g| < gradtol = 1 or the energy stalls), per-pose
segments.

`func(x)` must return (E [P] float64 or float32, g [P, L]).
"""

import torch


class LBFGSArmijo:
    def __init__(
        self,
        func,
        x0,
        max_iter=200,
        history_size=128,
        gradtol=1.0,
        rtol=None,
        c1=1e-4,
        shrink=0.5,
        max_linesearch=20,
    ):
        self.func = func
        self.x = x0.clone()
        self.max_iter = max_iter
        self.m = history_size
        self.gradtol = gradtol
        self.rtol = rtol if rtol is not None else float(torch.finfo(x0.dtype).eps ** 0.5)
        self.c1 = c1
        self.shrink = shrink
        self.max_ls = max_linesearch
        P, L = x0.shape
        dev, dt = x0.device, x0.dtype
        self.S = torch.zeros((history_size, P, L), device=dev, dtype=dt)
        self.Y = torch.zeros((history_size, P, L), device=dev, dtype=dt)
        # inner products between stored pairs, in slot order: [P, m, m]
        self.SY = torch.zeros((P, history_size, history_size), device=dev, dtype=torch.float64)
        self.YY = torch.zeros((P, history_size, history_size), device=dev, dtype=torch.float64)
        self.n_hist = 0
        self.head = 0
        self.n_evals = 0
        self.history = []

    def _direction(self, g):
        """-H g by the compact representation, per pose."""
        k = self.n_hist
        gd = g.double()
        if k == 0:
            gn = gd.norm(dim=-1)
            gamma = torch.where(gn > 0, 1.0 / gn, torch.ones_like(gn))
            return (-gamma[:, None] * gd).to(g.dtype)
        idx = torch.tensor(
            [(self.head - k + i) % self.m for i in range(k)], device=g.device, dtype=torch.long
        )
        S = self.S[idx].double()  # [k, P, L], oldest first
        Y = self.Y[idx].double()
        SY = self.SY[:, idx][:, :, idx]  # [P, k, k]
        YY = self.YY[:, idx][:, :, idx]
        D = SY.diagonal(dim1=-2, dim2=-1)
        newest = k - 1
        yy = YY[:, newest, newest]
        gamma = torch.where(yy > 0, D[:, newest] / yy, torch.ones_like(yy))
        R = torch.triu(SY)
        # empty pairs (poses that did not move) keep R invertible
        R = R + torch.diag_embed((D == 0).to(R.dtype))
        a = torch.einsum("kpl,pl->pk", S, gd)
        b = torch.einsum("kpl,pl->pk", Y, gd)
        v = torch.linalg.solve_triangular(R, a.unsqueeze(-1), upper=True).squeeze(-1)
        rhs = D * v + gamma[:, None] * torch.einsum("pij,pj->pi", YY, v) - gamma[:, None] * b
        top = torch.linalg.solve_triangular(R.transpose(-2, -1), rhs.unsqueeze(-1), upper=False).squeeze(-1)
        Hg = gamma[:, None] * gd + torch.einsum("pk,kpl->pl", top, S) - gamma[:, None] * torch.einsum("pk,kpl->pl", v, Y)
        return (-Hg).to(g.dtype)

    def _store(self, s, y):
        j = self.head
        self.S[j] = s
        self.Y[j] = y
        sd, yd = s.double(), y.double()
        Sd, Yd = self.S.double(), self.Y.double()
        self.SY[:, j, :] = torch.einsum("pl,mpl->pm", sd, Yd)
        self.SY[:, :, j] = torch.einsum("mpl,pl->pm", Sd, yd)
        yyj = torch.einsum("pl,mpl->pm", yd, Yd)
        self.YY[:, j, :] = yyj
        self.YY[:, :, j] = yyj
        self.head = (self.head + 1) % self.m
        self.n_hist = min(self.n_hist + 1, self.m)

    def run(self):
        x = self.x
        E, g = self.func(x)
        self.n_evals += 1
        E = E.double()
        P = x.shape[0]
        active = torch.ones(P, dtype=torch.bool, device=x.device)
        self.history.append(E.clone())
        for it in range(self.max_iter):
            gmax = g.abs().amax(-1)
            active &= gmax >= self.gradtol
            if not bool(active.any()):
                break
            d = self._direction(g)
            d = torch.where(active[:, None], d, torch.zeros_like(d))
            gd = (g.double() * d.double()).sum(-1)
            # an ascent direction (curvature lost): restart from steepest descent
            bad = gd >= 0
            if bool(bad.any()):
                d = torch.where(bad[:, None], -g, d)
                gd = torch.where(bad, -(g.double() ** 2).sum(-1), gd)
            t = torch.ones(P, dtype=torch.float64, device=x.device)
            accepted = ~active
            E_new = E.clone()
            x_new = x.clone()
            g_new = g.clone()
            for _ in range(self.max_ls):
                trial = x + (t.to(x.dtype))[:, None] * d
                Et, gt = self.func(trial)
                self.n_evals += 1
                Et = Et.double()
                ok = (~accepted) & (Et <= E + self.c1 * t * gd)
                x_new = torch.where(ok[:, None], trial, x_new)
                g_new = torch.where(ok[:, None], gt, g_new)
                E_new = torch.where(ok, Et, E_new)
                accepted |= ok
                if bool(accepted.all()):
                    break
                t = torch.where(accepted, t, t * self.shrink)
            # poses whose line search failed stop moving
            failed = ~accepted
            active &= ~failed
            s = x_new - x
            y = g_new - g
            sy = (s.double() * y.double()).sum(-1)
            keep = active & (sy > 1e-12)
            self._store(
                torch.where(keep[:, None], s, torch.zeros_like(s)),
                torch.where(keep[:, None], y, torch.zeros_like(y)),
            )
            dE = (E - E_new).abs()
            stalled = dE <= self.rtol * (E.abs() + E_new.abs() + 1.0) * 0.5
            x, g, E = x_new, g_new, E_new
            active &= ~stalled
            self.history.append(E.clone())
        self.x = x
        return x, E, g
