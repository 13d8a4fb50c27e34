"""The drop-in ops registered with torch's dispatcher.

tmol reaches its compiled scoring ops through ``torch.ops``:
``torch.ops.tmol_ljlk.ljlk_pose_scores`` / ``ljlk_rotamer_scores``
(``tmol/score/ljlk/potentials/compiled.ops.cpp:667-670``, bound in
``compiled.py:16-17``), ``torch.ops.tmol_elec.elec_pose_scores`` /
``elec_rotamer_scores`` (``tmol/score/elec/potentials/compiled.ops.cpp:
650-654``) and ``torch.ops.tmol_lk_ball.gen_pose_waters`` /
``lk_ball_pose_score`` / ``lk_ball_rotamer_score``
(``tmol/score/lk_ball/potentials/compiled.ops.cpp:978-982``).  Importing
this module defines the same seven ops, with the same schemas (argument
names, order and types, ``Tensor[]`` / ``Tensor`` results), under the
``tmol_b200`` namespace: ``torch.ops.tmol_b200.ljlk_pose_scores(...)``.

Each op is registered as a CompositeImplicitAutograd kernel over the
Python drop-ins in ``ljlk_op``, ``elec_op`` and ``lkball_op``, so autograd
runs through their ``torch.autograd.Function``s and the B200 adjoint
kernels (gradients for the coordinates and, for ``lk_ball_pose_score``,
the waters), exactly as when the drop-ins are called directly.  Like the
drop-ins, the ops take CUDA tensors only and raise otherwise.

``register_reference_aliases()`` (opt-in) also defines the ops under
tmol's own namespaces (``tmol_ljlk``, ``tmol_elec``, ``tmol_lk_ball``), so
that an installed tmol whose compiled extensions are not loaded reaches
these kernels without code changes.  It refuses a namespace whose ops are
already defined (tmol's own extension loaded in the same process).
"""

import torch

_COMMON = (
    "Tensor rot_coords, Tensor rot_coord_offset, Tensor pose_ind_for_atom, Tensor first_rot_for_block, "
    "Tensor first_rot_block_type, Tensor block_ind_for_rot, Tensor pose_ind_for_rot, "
    "Tensor block_type_ind_for_rot, Tensor n_rots_for_pose, Tensor rot_offset_for_pose, "
    "Tensor n_rots_for_block, Tensor rot_offset_for_block, int max_n_rots_per_pose"
)

# compiled.ops.cpp:533-560 (pose) and :599-626 (rotamer) of tmol/score/ljlk
_LJLK_ARGS = (
    _COMMON + ", Tensor pose_stack_min_bond_separation, Tensor pose_stack_inter_block_bondsep, "
    "Tensor block_type_n_atoms, Tensor block_type_n_heavy_atoms_in_tile, Tensor block_type_heavy_atoms_in_tile, "
    "Tensor block_type_atom_types, Tensor block_type_n_interblock_bonds, "
    "Tensor block_type_atoms_forming_chemical_bonds, Tensor block_type_path_distance, "
    "Tensor block_type_is_ligand_fragment, Tensor ljlk_type_params, Tensor global_params, float max_dis, "
    "bool output_block_pair_energies"
)

# tmol/score/elec/potentials/compiled.ops.cpp:526-552 and :588-614
_ELEC_ARGS = (
    _COMMON + ", Tensor pose_stack_min_bond_separation, Tensor pose_stack_inter_block_bondsep, "
    "Tensor block_type_n_atoms, Tensor block_type_partial_charge, Tensor block_type_n_interblock_bonds, "
    "Tensor block_type_atoms_forming_chemical_bonds, Tensor block_type_inter_repr_path_distance, "
    "Tensor block_type_intra_repr_path_distance, Tensor block_type_is_ligand_fragment, Tensor global_params, "
    "float max_dis, bool output_block_pair_energies"
)

# tmol/score/lk_ball/potentials/compiled.ops.cpp:283-318 (waters),
# :840-870 (pose score) and :909-939 (rotamer score)
_WATER_ARGS = (
    _COMMON + ", Tensor pose_stack_inter_residue_connections, Tensor block_type_n_atoms, "
    "Tensor block_type_n_interblock_bonds, Tensor block_type_atoms_forming_chemical_bonds, "
    "Tensor block_type_n_all_bonds, Tensor block_type_all_bonds, Tensor block_type_atom_all_bond_ranges, "
    "Tensor block_type_tile_n_donH, Tensor block_type_tile_n_acc, Tensor block_type_tile_donH_inds, "
    "Tensor block_type_tile_don_hvy_inds, Tensor block_type_tile_which_donH_for_hvy, "
    "Tensor block_type_tile_acc_inds, Tensor block_type_tile_hybridization, "
    "Tensor block_type_tile_acc_n_attached_H, Tensor block_type_atom_is_hydrogen, Tensor global_params, "
    "Tensor sp2_water_tors, Tensor sp3_water_tors, Tensor ring_water_tors"
)
_LKB_SCORE_ARGS = (
    _COMMON + ", Tensor pose_stack_inter_residue_connections, Tensor pose_stack_min_bond_separation, "
    "Tensor pose_stack_inter_block_bondsep, Tensor block_type_n_atoms, Tensor block_type_n_interblock_bonds, "
    "Tensor block_type_atoms_forming_chemical_bonds, Tensor block_type_tile_n_polar_atoms, "
    "Tensor block_type_tile_n_occluder_atoms, Tensor block_type_tile_pol_occ_inds, "
    "Tensor block_type_tile_lk_ball_params, Tensor block_type_path_distance, Tensor global_params, "
    "float max_dis, Tensor water_coords, bool output_block_pair_energies"
)


def _ljlk_pose_scores(*args):
    from .ljlk_op import ljlk_pose_scores

    E, nbr = ljlk_pose_scores(*args)
    return [E, nbr]


def _ljlk_rotamer_scores(*args):
    from .ljlk_op import ljlk_rotamer_scores

    return list(ljlk_rotamer_scores(*args))


def _elec_pose_scores(*args):
    from .elec_op import elec_pose_scores

    E, nbr = elec_pose_scores(*args)
    return [E, nbr]


def _elec_rotamer_scores(*args):
    from .elec_op import elec_rotamer_scores

    return list(elec_rotamer_scores(*args))


def _gen_pose_waters(*args):
    from .lkball_op import gen_pose_waters

    return gen_pose_waters(*args)


def _lk_ball_pose_score(*args):
    from .lkball_op import lk_ball_pose_score

    E, nbr = lk_ball_pose_score(*args)
    return [E, nbr]


def _lk_ball_rotamer_score(*args):
    from .lkball_op import lk_ball_rotamer_score

    return list(lk_ball_rotamer_score(*args))


# namespace of the reference's extension -> (op name, argument list, result, implementation)
OPS = {
    "tmol_ljlk": [
        ("ljlk_pose_scores", _LJLK_ARGS, "Tensor[]", _ljlk_pose_scores),
        ("ljlk_rotamer_scores", _LJLK_ARGS, "Tensor[]", _ljlk_rotamer_scores),
    ],
    "tmol_elec": [
        ("elec_pose_scores", _ELEC_ARGS, "Tensor[]", _elec_pose_scores),
        ("elec_rotamer_scores", _ELEC_ARGS, "Tensor[]", _elec_rotamer_scores),
    ],
    "tmol_lk_ball": [
        ("gen_pose_waters", _WATER_ARGS, "Tensor", _gen_pose_waters),
        ("lk_ball_pose_score", _LKB_SCORE_ARGS, "Tensor[]", _lk_ball_pose_score),
        ("lk_ball_rotamer_score", _LKB_SCORE_ARGS, "Tensor[]", _lk_ball_rotamer_score),
    ],
}

NAMESPACE = "tmol_b200"
_LIBS = {}


def _defined(ns, name):
    try:
        getattr(getattr(torch.ops, ns), name)
        return True
    except (AttributeError, RuntimeError):
        return False


def _register(ns, ops):
    lib = torch.library.Library(ns, "FRAGMENT")
    for name, args, result, impl in ops:
        lib.define(f"{name}({args}) -> {result}")
        lib.impl(name, impl, "CompositeImplicitAutograd")
    _LIBS[ns] = lib


def register():
    """Defines the seven ops under ``tmol_b200`` (idempotent)."""
    if NAMESPACE in _LIBS:
        return
    _register(NAMESPACE, [op for ops in OPS.values() for op in ops])


def register_reference_aliases():
    """Defines the ops under tmol's own namespaces as well; returns the
    namespaces registered.  Raises if one of them already has its ops."""
    register()
    done = []
    for ns, ops in OPS.items():
        if ns in _LIBS:
            done.append(ns)
            continue
        taken = [name for name, *_ in ops if _defined(ns, name)]
        if taken:
            raise RuntimeError(f"torch.ops.{ns} already defines {taken}: tmol's own extension is loaded")
        _register(ns, ops)
        done.append(ns)
    return done


register()
