"""``run_min``: minimise a scoring module with a closure-driven optimiser,
tmol's ``tmol/optimization/minimizers.py:54-126``: per-pose segments when
the module provides ``segment_ids`` and the optimiser supports them; the
closure zeroes the gradient, scores, backpropagates the summed energies and
returns the per-pose energies.  Returns the minimised PoseStack and the
optimiser (its ``n_evals`` and ``energy_history`` describe the run)."""

from .lbfgs_armijo import LBFGS_Armijo


def run_min(sfxn_module, optimizer_cls=LBFGS_Armijo, optimizer_kwargs=None, per_pose=True):
    kwargs = dict(optimizer_kwargs or {})
    seg = getattr(sfxn_module, "segment_ids", None)
    segmented = per_pose and seg is not None and getattr(optimizer_cls, "supports_segments", False)
    if segmented:
        kwargs["segment_ids"] = seg
    opt = optimizer_cls(sfxn_module.parameters(), **kwargs)

    def closure():
        opt.zero_grad()
        E = sfxn_module()
        E.sum().backward()
        return E if segmented else E.sum()

    opt.step(closure)
    return sfxn_module.pose_stack_from_dofs(), opt
