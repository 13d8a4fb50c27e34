"""``LBFGS_Armijo``: tmol's minimiser, with tmol's interface, for driving the
B200 scoring ops exactly as tmol drives its own.

tmol minimises with ``tmol.optimization.lbfgs_armijo.LBFGS_Armijo``
(``tmol/optimization/lbfgs_armijo.py:196-744``), a ``torch.optim.Optimizer``
whose single ``step(closure)`` runs a whole minimisation: limited-memory
BFGS with Rosetta's Armijo line search, optionally split into independent
segments (one per pose) that share every function evaluation.  This module
states that algorithm over the same interface (constructor arguments,
``supports_segments``, per-segment closures returning one energy per
segment), so that tmol's ``run_min`` and ``CartesianSfxnNetwork``
(``tmol/optimization/minimizers.py:54-126``, ``sfxn_modules.py:12-69``) run
unchanged over the B200 ops, and so that a minimisation here takes the same
steps as tmol's on the same energies (checked against tmol's own class and
its stored trajectories in the tests).

The steps, with the reference lines they follow:

* search direction (``lbfgs_armijo.py:467-534``): steepest descent on the
  first iteration; afterwards the pair (y, s) = (g - g_prev, x - x_ref) is
  stored for the segments whose curvature y.s exceeds 1e-6 (x_ref then moves
  to x), in a ring of ``history_size`` pairs, and the direction is the
  compact-representation product -H g with H0 = I (Byrd, Nocedal &
  Schnabel 1994; ``lbfgs_two_loop``, ``:6-57``), solved in float64 per
  segment;
* a segment whose line search failed restarts from steepest descent with
  its history dropped (``:536-554``); converged or retired segments do not
  move (``:560-566``);
* the directional derivative g.d is repaired where it is not below -1e-5:
  first by flipping the sign of the components that point uphill, then by
  falling back to -g (``:568-587``);
* the line search (``armijo_linesearch_segmented``, ``:66-193``; Bertsekas,
  Nonlinear Programming, p. 29): each segment starts from twice its last
  accepted step, at most 1; a step whose decrease looks linear
  (sigma 0.8) is tried once at twice the length and kept if better; a
  step without sufficient decrease (sigma 0.1) shrinks by 0.25 until it has
  it; below ``minstep`` any decrease is accepted, else the search fails
  (the step restarts at min(1, 1/sqrt|g.d|), ``:589-628``);
* convergence (``:630-670``): a segment freezes once max|g| <= ``gradtol``;
  the run ends when every segment is frozen, retired, or changed its energy
  by at most ``atol`` or ``rtol`` (relative) in the last iteration.
"""

import torch
from torch.optim import Optimizer

# line-search state of a segment
_DONE, _LONGER, _SHORTER, _FAILED = 0, 1, 2, 3


class _Segments:
    """Element -> segment bookkeeping: a parameter-shaped vector scattered
    into a dense [n_segments, segment_size] block (zero padding) for the
    per-segment sums, maxima and the batched direction solve."""

    def __init__(self, seg):
        seg = seg.reshape(-1).to(torch.int64)
        if bool((seg < 0).any()):
            raise ValueError("segment_ids must be non-negative")
        self.seg = seg
        self.n = int(seg.max().item()) + 1 if seg.numel() else 1
        counts = torch.bincount(seg, minlength=self.n)
        if bool((counts == 0).any()):
            raise ValueError("segment_ids must not skip a segment")
        self.size = int(counts.max().item())
        order = torch.argsort(seg, stable=True)
        start = torch.cumsum(counts, 0) - counts
        rank = torch.empty_like(order)
        rank[order] = torch.arange(seg.numel(), device=seg.device) - start[seg[order]]
        self.slot = seg * self.size + rank

    def pad(self, v, out=None):
        if out is None:
            out = torch.zeros(self.n * self.size, dtype=v.dtype, device=v.device)
        else:
            out = out.view(-1)
            out.zero_()
        out[self.slot] = v
        return out.view(self.n, self.size)

    def unpad(self, block):
        return block.reshape(-1)[self.slot]

    def sum(self, v):
        return self.pad(v).sum(-1)

    def amax(self, v):
        out = torch.empty(self.n, dtype=v.dtype, device=v.device)
        return out.scatter_reduce_(0, self.seg, v, "amax", include_self=False)

    def expand(self, per_segment):
        return per_segment[self.seg]


def compact_direction(grad, Y, S):
    """-H grad for each segment, with H the L-BFGS inverse Hessian of the
    stored pairs (H0 = I) in compact form: with q = -grad, a = S q, b = Y q,
    R = upper(S Y^T) (unit diagonal where a slot is empty), D = diag(S Y^T),
    u = R^-1 a, the direction is q + S^T R^-T ((D + Y Y^T) u - b) - Y^T u.
    grad [k, n]; Y, S [m, k, n] (oldest first).  Computed in float64."""
    S64, Y64 = S.double(), Y.double()
    q = -grad.double()
    a = torch.einsum("ipk,pk->pi", S64, q)
    b = torch.einsum("ipk,pk->pi", Y64, q)
    SY = torch.einsum("ipk,jpk->pij", S64, Y64)
    YY = torch.einsum("ipk,jpk->pij", Y64, Y64)
    D = SY.diagonal(dim1=-2, dim2=-1)
    R = torch.triu(SY) + torch.diag_embed((D == 0).to(SY.dtype))
    u = torch.linalg.solve_triangular(R, a.unsqueeze(-1), upper=True).squeeze(-1)
    w = torch.einsum("pij,pj->pi", YY, u) + D * u - b
    r = torch.linalg.solve_triangular(R.transpose(-2, -1), w.unsqueeze(-1), upper=False).squeeze(-1)
    d = q + torch.einsum("pi,ipk->pk", r, S64) + torch.einsum("pi,ipk->pk", -u, Y64)
    return d.to(grad.dtype)


def segmented_armijo(phi_of, slope, phi0, alpha0, active, shrink=0.5, sigma_sufficient=0.1,
                     sigma_linear=0.8, minstep=1e-6):
    """Rosetta's Armijo search, one step length per segment, every trial
    evaluating all segments at once through ``phi_of(alphas)``.  Returns
    (accepted steps, their energies, evaluations, final states, whether the
    last evaluation was at the accepted steps)."""
    zero = torch.zeros_like(alpha0)
    alpha = torch.where(active, alpha0, zero)
    taken = zero.clone()
    phi_taken = phi0.clone()
    state = torch.full(alpha0.shape, _DONE, dtype=torch.int64, device=alpha0.device)
    phi = phi_of(alpha)
    evals = 1
    looks_linear = phi <= phi0 + alpha * sigma_linear * slope
    decreased = phi <= phi0 + alpha * sigma_sufficient * slope
    state = torch.where(active & looks_linear, _LONGER, state)
    state = torch.where(active & ~looks_linear & ~decreased, _SHORTER, state)
    ok = active & (looks_linear | decreased)
    taken = torch.where(ok, alpha, taken)
    phi_taken = torch.where(ok, phi, phi_taken)
    while bool(((state == _LONGER) | (state == _SHORTER)).any()):
        longer, shorter = state == _LONGER, state == _SHORTER
        trial = torch.where(longer, alpha / shrink, taken)
        trial = torch.where(shorter, alpha * shrink * shrink, trial)
        phi_trial = phi_of(trial)
        evals += 1
        # a longer step is kept only if it beats the one already taken
        better = longer & (phi_trial < phi)
        taken = torch.where(better, trial, taken)
        phi_taken = torch.where(better, phi_trial, phi_taken)
        state = torch.where(longer, _DONE, state)
        # a shorter step until the decrease is sufficient
        suff = shorter & (phi_trial <= phi0 + trial * sigma_sufficient * slope)
        taken = torch.where(suff, trial, taken)
        phi_taken = torch.where(suff, phi_trial, phi_taken)
        state = torch.where(suff, _DONE, state)
        # below the smallest step: any decrease, else a failed search
        tiny = shorter & ~suff & (trial < minstep)
        down = tiny & (phi_trial < phi0)
        taken = torch.where(down, trial, taken)
        phi_taken = torch.where(down, phi_trial, phi_taken)
        state = torch.where(down, _DONE, state)
        fail = tiny & ~down
        taken = torch.where(fail, zero, taken)
        phi_taken = torch.where(fail, phi0, phi_taken)
        state = torch.where(fail, _FAILED, state)
        alpha, phi = trial, phi_trial
    return taken, phi_taken, evals, state, bool(torch.equal(alpha, taken))


class LBFGS_Armijo(Optimizer):
    """L-BFGS with Armijo line search; tmol's constructor and ``step``.

    Parameters (tmol's): ``lr`` the first iteration's step (1), ``max_iter``
    (200), ``rtol`` / ``atol`` energy-change tolerances (default: the square
    root of the parameter dtype's epsilon), ``gradtol`` on max |dE/dx| (1),
    ``history_size`` (128), ``minstep`` (1e-12), ``verbose``,
    ``segment_ids`` (the segment, e.g. pose, of each parameter element;
    segments are minimised independently)."""

    supports_segments = True

    def __init__(self, params, lr=1, max_iter=200, rtol=None, atol=None, gradtol=1.0, history_size=128,
                 minstep=1e-12, verbose=False, segment_ids=None):
        super().__init__(params, dict(lr=lr, max_iter=max_iter, atol=atol, rtol=rtol, gradtol=gradtol,
                                      history_size=history_size))
        if len(self.param_groups) != 1 or len(self.param_groups[0]["params"]) != 1:
            raise ValueError("LBFGS_Armijo takes a single parameter tensor")
        self._param = self.param_groups[0]["params"][0]
        self._minstep = minstep
        self.verbose = verbose
        if segment_ids is None:
            segment_ids = torch.zeros(self._param.numel(), dtype=torch.int64, device=self._param.device)
        if segment_ids.numel() != self._param.numel():
            raise ValueError("segment_ids needs one entry per parameter element")
        self._segs = _Segments(segment_ids.to(self._param.device))
        self._energies = None
        self.n_evals = 0
        self.energy_history = []

    # -- evaluation ---------------------------------------------------------

    def _evaluate(self, closure):
        """Calls the closure; keeps its per-segment energies."""
        loss = closure()
        self.n_evals += 1
        if torch.is_tensor(loss) and loss.numel() == self._segs.n:
            self._energies = loss.detach().reshape(self._segs.n)
        else:
            self._energies = torch.as_tensor(loss).detach().reshape(1).expand(self._segs.n).clone()
        return self._energies

    def step(self, closure):
        """Minimises from the parameter's current value; returns the first
        evaluation's result, as tmol's ``step`` does."""
        group = self.param_groups[0]
        P = self._param
        segs = self._segs
        eps_tol = float(torch.finfo(P.dtype).eps ** 0.5)
        rtol = eps_tol if group["rtol"] is None else group["rtol"]
        atol = eps_tol if group["atol"] is None else group["atol"]
        m = group["history_size"]
        st = self.state[P]
        st.setdefault("n_iter", 0)

        first = closure()
        self.n_evals += 1
        if torch.is_tensor(first) and first.numel() == segs.n:
            self._energies = first.detach().reshape(segs.n)
        else:
            self._energies = torch.as_tensor(first).detach().reshape(1).expand(segs.n).clone()
        energies = self._energies
        self.energy_history.append(energies.clone())
        x = P.data.view(-1)
        g = P.grad.data.view(-1)
        if "d" not in st:
            flags = dict(dtype=torch.bool, device=x.device)
            st.update(
                d=torch.empty_like(x), x0=torch.empty_like(x), x_ref=x.clone(),
                Y=torch.zeros((m, segs.n, segs.size), dtype=x.dtype, device=x.device),
                S=torch.zeros((m, segs.n, segs.size), dtype=x.dtype, device=x.device),
                g_pad=torch.zeros((segs.n, segs.size), dtype=x.dtype, device=x.device),
                count=0, start=0,
                converged=torch.zeros(segs.n, **flags), retired=torch.zeros(segs.n, **flags),
                restart=torch.zeros(segs.n, **flags), restarted=torch.zeros(segs.n, **flags),
                t=None, g_prev=None, e_prev=None,
            )
        d, x0 = st["d"], st["x0"]

        def phi_of(alphas):
            x.copy_(x0).add_(d * segs.expand(alphas))
            return self._evaluate(closure)

        for it in range(group["max_iter"]):
            st["n_iter"] += 1
            frozen = st["converged"] | st["retired"]
            # direction
            if st["n_iter"] == 1:
                d.copy_(g).neg_()
                st["count"] = 0
            else:
                y = g - st["g_prev"]
                s = x - st["x_ref"]
                curved = segs.sum(y * s) > 1e-6
                if bool(curved.any()):
                    if st["count"] < m:
                        slot = st["count"]
                        st["count"] += 1
                    else:
                        slot = st["start"]
                        st["start"] = (st["start"] + 1) % m
                    keep = segs.expand(curved)
                    z = torch.zeros((), dtype=x.dtype, device=x.device)
                    segs.pad(torch.where(keep, y, z), out=st["Y"][slot])
                    segs.pad(torch.where(keep, s, z), out=st["S"][slot])
                    st["x_ref"] = torch.where(keep, x, st["x_ref"])
                if st["count"] == 0:
                    d.copy_(g).neg_()
                else:
                    if st["count"] < m:
                        Yv, Sv = st["Y"][: st["count"]], st["S"][: st["count"]]
                    else:
                        order = torch.cat([torch.arange(st["start"], m, device=x.device),
                                           torch.arange(0, st["start"], device=x.device)])
                        Yv, Sv = st["Y"][order], st["S"][order]
                    d.copy_(segs.unpad(compact_direction(segs.pad(g, out=st["g_pad"]), Yv, Sv)))
            # a failed search restarts its segment from steepest descent
            if bool(st["restart"].any()):
                st["restarted"] = st["restart"].clone()
                idx = st["restart"].nonzero(as_tuple=False).squeeze(-1)
                st["Y"][:, idx, :] = 0.0
                st["S"][:, idx, :] = 0.0
                r = segs.expand(st["restart"])
                d.copy_(torch.where(r, -g, d))
                st["x_ref"] = torch.where(r, x, st["x_ref"])
                st["restart"] = torch.zeros_like(st["restart"])
            else:
                st["restarted"] = torch.zeros_like(st["restart"])
            if bool(frozen.any()):
                d.mul_(segs.expand(~frozen).to(d.dtype))
            if st["g_prev"] is None:
                st["g_prev"] = g.clone()
            else:
                st["g_prev"].copy_(g)
            e_before = energies
            if st["n_iter"] == 1:
                st["t"] = torch.full((segs.n,), float(group["lr"]), dtype=x.dtype, device=x.device)
            # downhill slope, repaired where it is not
            slope = segs.sum(g * d)
            for repair in (1, 2):
                uphill = (slope > -1e-5) & ~frozen
                if not bool(uphill.any()):
                    break
                fixed = d * -torch.sign(g * d) if repair == 1 else -g
                d.copy_(torch.where(segs.expand(uphill), fixed, d))
                slope = segs.sum(g * d)
            # line search from x0, each segment from twice its last step
            x0.copy_(x)
            active = ~frozen & (slope < 0)
            t0 = (st["t"] / 0.5).clamp(max=1.0)
            taken, _, _, state, at_taken = segmented_armijo(
                phi_of, slope, e_before, t0, active, shrink=0.5, sigma_sufficient=0.1, sigma_linear=0.8,
                minstep=self._minstep,
            )
            x.copy_(x0).add_(d * segs.expand(taken))
            if not at_taken:
                self._evaluate(closure)
            energies = self._energies
            failed = state == _FAILED
            retry = torch.clamp((-slope).clamp(min=self._minstep).rsqrt(), max=1.0)
            st["t"] = torch.where(active, torch.where(failed, retry, taken), t0)
            if bool(failed.any()):
                if self.verbose:
                    print(f"line search failed on segments {failed.nonzero().flatten().tolist()}")
                st["retired"] |= failed & st["restarted"]
                st["restart"] |= failed & ~st["restarted"]
            g = P.grad.data.view(-1)
            self.energy_history.append(energies.clone())
            # convergence
            st["converged"] |= segs.amax(g.abs()) <= group["gradtol"]
            finished = st["converged"] | st["retired"]
            dE = (energies - e_before).abs()
            rel = 2 * dE / (energies.abs() + e_before.abs() + 1e-10)
            finished = finished | (dE <= atol) | (rel <= rtol)
            if self.verbose:
                print(f"  iter {it + 1:4d}  E={float(energies.sum()):.6f}  done={int(finished.sum())}/{segs.n}")
            if bool(finished.all()):
                break
        st["e_prev"] = energies
        return first
