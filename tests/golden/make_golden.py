"""Generate the golden fixtures under tests/golden from the reference itself.

Run in a checkout that has the reference sources and the compiled reference
op (``python oracle/build_ref.py``):

    python tests/golden/make_golden.py /path/to/tmol

Writes
  ubq.npz            1ubq (tmol/tests/data/pdb/1ubq.pdb) as block-type names
                     and coordinates in block-type atom order, the reference
                     op's per-pose energies and gradient for it, and the
                     reference test suite's stored whole-pose energies
                     (tmol/tests/data/term_baselines/LJLKEnergyTerm/
                     test_whole_pose_scoring_10.yaml)
  ubq_blockpair.npz  reference op block-pair energies of 1ubq
  synthetic.npz      reference op energies, gradient and neighbour matrix of
                     a jagged batch of seeded synthetic poses (1, 2, 7, 33,
                     100 residues), plus the sizes and seeds that rebuild it
  elec.npz           the reference elec op (elec_pose_scores) on 1ubq and on
                     a jagged synthetic batch: per-pose energies, gradient,
                     neighbour matrix and block-pair energies, plus the
                     reference test suite's stored 1ubq elec energy
                     (tmol/tests/data/term_baselines/ElecEnergyTerm/
                     test_whole_pose_scoring_10.yaml); and the
                     reference elec rotamer op (elec_rotamer_scores) on the
                     rotamer set of rotamers.npz (energies, indices, the
                     gradient of sum(w * E) for seeded w)
  lkball.npz         the reference LK-ball ops (gen_pose_waters, then
                     lk_ball_pose_score) on 1ubq and on a seeded synthetic
                     pose, float32 and float64: waters, the four energies,
                     the gradient of their sum; plus the reference test
                     suite's stored 1ubq LK-ball energies
                     (tmol/tests/data/term_baselines/LKBallEnergyTerm/
                     test_whole_pose_scoring_10.yaml)
  lkball_rotamers.npz  the reference LK-ball rotamer op (gen_pose_waters on the
                     rotamers' coordinates, then lk_ball_rotamer_score) on
                     the rotamer set of rotamers.npz, float32 and float64:
                     waters, rotamer-pair energies, dispatch indices and the
                     gradient of sum(w * E) for seeded w
                     (``make_golden.py <tmol root> lkball_rotamers`` writes
                     this file alone)
  lkball_block_pair.npz  the reference lk_ball_pose_score in block-pair mode
                     on the synthetic pose of lkball.npz, float32 and
                     float64: energies [4, P, B, B] and the gradient of
                     sum(w * E) for seeded w (``... lkball_block_pair``
                     writes this file alone)
  rotamers.npz       the reference rotamer-score op (ljlk_rotamer_scores) on
                     a seeded rotamer set over a jagged batch of poses: the
                     set itself, the rotamer-pair energies and dispatch
                     indices, and the gradient of sum(w * E) for seeded w
"""

import os
import sys

import numpy
import torch
import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle import oracle as O  # noqa: E402
from tmol_b200.pose.builder import build_pose_stack  # noqa: E402
from tmol_b200.pose.pdb import pose_from_pdb_text  # noqa: E402
from tmol_b200.pose.synthetic import synthetic_pose_stack  # noqa: E402
from tmol_b200.pose.rotamers import synthetic_rotamer_set  # noqa: E402
from tmol_b200.score.elec_energy_term import (  # noqa: E402
    ElecEnergyTerm,
    elec_pose_score_args,
    elec_rotamer_score_args,
)
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args, rotamer_score_args  # noqa: E402
from tmol_b200.score.lkball_energy_term import (  # noqa: E402
    LKBallEnergyTerm,
    rotamer_score_args as lkball_rotamer_score_args,
    score_args,
    water_gen_args,
)

SYN_SIZES = [1, 2, 7, 33, 100]
SYN_SEEDS = [11, 12, 13, 14, 15]
ELEC_SIZES = [40, 3, 17, 120]
ELEC_SEEDS = [31, 32, 33, 34]
LKB_SYN = ([60], [44], 20.0)  # sizes, seeds, extra chi sd
ROT_SIZES = [12, 30, 1, 45]
ROT_SEEDS = [21, 22, 23, 24]
ROT_SET = dict(max_rots=4, mutate_fraction=0.25, seed=5, skip_fraction=0.1)
ROT_FIELDS = (
    "n_rots_for_pose", "rot_offset_for_pose", "n_rots_for_block", "rot_offset_for_block", "pose_for_rot",
    "block_type_ind_for_rot", "block_ind_for_rot", "coord_offset_for_rot", "coords", "first_rot_block_type",
    "pose_ind_for_atom",
)


def ref_scores(ps, term):
    args = pose_score_args(ps, term)
    coords = ps.coords.flatten(0, 1)
    E, c, nbr = O.reference_pose_scores(coords, args, require_gradient=True)
    E.sum().backward()
    return E.detach().numpy(), c.grad.numpy(), nbr.numpy()


def main(ref_root):
    term = LJLKEnergyTerm()
    with open(os.path.join(ref_root, "tmol/tests/data/pdb/1ubq.pdb")) as f:
        topo, xyz = pose_from_pdb_text(f.read())
    with open(
        os.path.join(
            ref_root,
            "tmol/tests/data/term_baselines/LJLKEnergyTerm/test_whole_pose_scoring_10.yaml",
        )
    ) as f:
        gold = yaml.safe_load(f)
    gold_E = numpy.array([gold[f"term{t}"]["pose0"] for t in range(3)], dtype=numpy.float64)
    ps = build_pose_stack([topo], [xyz])
    E, g, nbr = ref_scores(ps, term)
    numpy.savez_compressed(
        os.path.join(HERE, "ubq.npz"),
        block_type_names=numpy.array(topo.block_type_names),
        coords=xyz.astype(numpy.float32),
        ref_energies=E,
        ref_grad=g,
        ref_neighbors=nbr,
        tmol_test_energies=gold_E,
    )
    args = pose_score_args(ps, term, block_pair=True)
    Eb, _ = O.load_reference()(ps.coords.flatten(0, 1).clone(), *args)
    numpy.savez_compressed(os.path.join(HERE, "ubq_blockpair.npz"), ref_block_pair_energies=Eb.numpy())

    ps = synthetic_pose_stack(SYN_SIZES, SYN_SEEDS)
    E, g, nbr = ref_scores(ps, term)
    numpy.savez_compressed(
        os.path.join(HERE, "synthetic.npz"),
        sizes=numpy.array(SYN_SIZES),
        seeds=numpy.array(SYN_SEEDS),
        coords=ps.coords.numpy(),
        ref_energies=E,
        ref_grad=g,
        ref_neighbors=nbr,
    )
    eterm = ElecEnergyTerm()
    with open(
        os.path.join(ref_root, "tmol/tests/data/term_baselines/ElecEnergyTerm/test_whole_pose_scoring_10.yaml")
    ) as f:
        elec_gold = yaml.safe_load(f)
    out = {"ubq_tmol_test_energy": numpy.array([elec_gold["term0"]["pose0"]], dtype=numpy.float64)}
    for tag, eps_ in (("ubq", build_pose_stack([topo], [xyz])), ("syn", synthetic_pose_stack(ELEC_SIZES, ELEC_SEEDS))):
        coords = eps_.coords.flatten(0, 1)
        E, c, nbr = O.reference_elec_pose_scores(coords, elec_pose_score_args(eps_, eterm), require_gradient=True)
        E.sum().backward()
        Eb, _, _ = O.reference_elec_pose_scores(coords, elec_pose_score_args(eps_, eterm, True), require_gradient=False)
        out.update({
            f"{tag}_energies": E.detach().numpy(),
            f"{tag}_grad": c.grad.numpy(),
            f"{tag}_neighbors": nbr.numpy(),
            f"{tag}_block_pair": Eb.detach().numpy(),
        })
    lterm = LKBallEnergyTerm()
    with open(
        os.path.join(ref_root, "tmol/tests/data/term_baselines/LKBallEnergyTerm/test_whole_pose_scoring_10.yaml")
    ) as f:
        lgold = yaml.safe_load(f)
    lout = {"ubq_tmol_test_energies": numpy.array([lgold[f"term{t}"]["pose0"] for t in range(4)], numpy.float64)}
    lsyn = synthetic_pose_stack(LKB_SYN[0], LKB_SYN[1], extra_chi_sd=LKB_SYN[2])
    for tag, lps in (("ubq", build_pose_stack([topo], [xyz])), ("syn", lsyn)):
        for dt, dn in ((torch.float32, "f32"), (torch.float64, "f64")):
            wa = water_gen_args(lps, lterm)
            sa = score_args(lps, lterm, None)
            if dt == torch.float64:
                wa = [a.to(dt) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in wa]
                sa = [a.to(dt) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in sa]
            E, W, c, _ = O.reference_lkball(lps.coords.flatten(0, 1).to(dt), wa, sa)
            E.sum().backward()
            lout[f"{tag}_{dn}_energies"] = E.detach().numpy()
            lout[f"{tag}_{dn}_waters"] = W.detach().numpy()
            lout[f"{tag}_{dn}_grad"] = c.grad.numpy()
    numpy.savez_compressed(
        os.path.join(HERE, "lkball.npz"),
        syn_sizes=numpy.array(LKB_SYN[0]),
        syn_seeds=numpy.array(LKB_SYN[1]),
        syn_chi_sd=numpy.array(LKB_SYN[2]),
        **lout,
    )

    ps = synthetic_pose_stack(ROT_SIZES, ROT_SEEDS)
    rs = synthetic_rotamer_set(ps, **ROT_SET)
    E, c, idx = O.reference_elec_rotamer_scores(rs.coords, elec_rotamer_score_args(ps, rs, eterm))
    w = torch.tensor(numpy.random.default_rng(9).normal(size=tuple(E.shape)), dtype=E.dtype)
    (E * w).sum().backward()
    out.update({
        "rot_energies": E.detach().numpy(),
        "rot_indices": idx.numpy(),
        "rot_weights": w.numpy(),
        "rot_grad": c.grad.numpy(),
    })
    numpy.savez_compressed(
        os.path.join(HERE, "elec.npz"), sizes=numpy.array(ELEC_SIZES), seeds=numpy.array(ELEC_SEEDS), **out
    )

    args = rotamer_score_args(ps, rs, term)
    E, c, idx = O.reference_rotamer_scores(rs.coords, args, require_gradient=True)
    w = torch.tensor(numpy.random.default_rng(7).normal(size=tuple(E.shape)), dtype=E.dtype)
    (E * w).sum().backward()
    numpy.savez_compressed(
        os.path.join(HERE, "rotamers.npz"),
        sizes=numpy.array(ROT_SIZES),
        seeds=numpy.array(ROT_SEEDS),
        pose_coords=ps.coords.numpy(),
        max_n_rots_per_pose=numpy.array(rs.max_n_rots_per_pose),
        **{f: getattr(rs, f).numpy() for f in ROT_FIELDS},
        ref_energies=E.detach().numpy(),
        ref_indices=idx.numpy(),
        weights=w.numpy(),
        ref_grad=c.grad.numpy(),
    )


def lkball_rotamers():
    """lkball_rotamers.npz (the rotamer set is rebuilt from its seeds, as
    rotamers.npz stores it)."""
    ps = synthetic_pose_stack(ROT_SIZES, ROT_SEEDS)
    rs = synthetic_rotamer_set(ps, **ROT_SET)
    lterm = LKBallEnergyTerm()
    out = {}
    for dt, dn in ((torch.float32, "f32"), (torch.float64, "f64")):
        wa = water_gen_args(ps, lterm, rs)
        sa = lkball_rotamer_score_args(ps, rs, lterm, None)
        wa = [a.to(dt) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in wa]
        sa = [a.to(dt) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in sa]
        E, idx, W, c = O.reference_lkball_rotamers(rs.coords.to(dt), wa, sa)
        w = torch.tensor(numpy.random.default_rng(11).normal(size=tuple(E.shape)), dtype=dt)
        (E * w).sum().backward()
        out.update({
            f"{dn}_energies": E.detach().numpy(),
            f"{dn}_waters": W.detach().numpy(),
            f"{dn}_weights": w.numpy(),
            f"{dn}_grad": c.grad.numpy(),
        })
        out["indices"] = idx.numpy()
    numpy.savez_compressed(os.path.join(HERE, "lkball_rotamers.npz"), **out)


def lkball_block_pair():
    """lkball_block_pair.npz"""
    ps = synthetic_pose_stack(LKB_SYN[0], LKB_SYN[1], extra_chi_sd=LKB_SYN[2])
    lterm = LKBallEnergyTerm()
    out = {}
    for dt, dn in ((torch.float32, "f32"), (torch.float64, "f64")):
        wa = water_gen_args(ps, lterm)
        sa = score_args(ps, lterm, None, block_pair=True)
        wa = [a.to(dt) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in wa]
        sa = [a.to(dt) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in sa]
        E, W, c, nbr = O.reference_lkball(ps.coords.flatten(0, 1).to(dt), wa, sa)
        w = torch.tensor(numpy.random.default_rng(12).normal(size=tuple(E.shape)), dtype=dt)
        (E * w).sum().backward()
        out.update({f"{dn}_energies": E.detach().numpy(), f"{dn}_weights": w.numpy(), f"{dn}_grad": c.grad.numpy()})
    numpy.savez_compressed(os.path.join(HERE, "lkball_block_pair.npz"), **out)


if __name__ == "__main__":
    from oracle.build_ref import reference_root

    root = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    only = sys.argv[2] if len(sys.argv) > 2 else None
    if only == "lkball_rotamers":
        lkball_rotamers()
    elif only == "lkball_block_pair":
        lkball_block_pair()
    else:
        main(root)
        lkball_rotamers()
        lkball_block_pair()
    print("wrote fixtures to", HERE)
