"""Extract the chemistry and LJ/LK parameter tables this package needs from a
tmol parameter database into one compact JSON file.

The LJ/LK energy is defined by tmol's database: atom types and their chemical
flags (``database/default/chemical/chemical.yaml``), residue types (atoms,
bonds, inter-residue connections, internal coordinates, torsions) and the
LJ/LK parameters (``database/default/scoring/ljlk.yaml``).  Scoring the same
chemistry requires the same numbers, so they are read from tmol's files rather
than retyped.  The output keeps only what the LJ/LK path and the synthetic
pose builder use:

* every atom type (name, element, donor/acceptor/hydroxyl/polar-H flags) in
  the order ``chemical.yaml`` lists them, joined with its ``ljlk.yaml`` row
  (``tmol/score/ljlk/params.py:99-163`` performs the same join);
* the canonical L-amino-acid residue types plus HIS_D;
* the LJ/LK global parameters, and the LK-ball water-placement ones
  (``lkb_water_*``; angles converted to radians as tmol's unit parser does);
* the hbond donor and acceptor atom types (``database/default/scoring/
  hbond.yaml``: which atom types donate or accept, as the LK-ball term builds
  waters on them) and each atom type's acceptor hybridization
  (``chemical.yaml``).

The elec term's parameters (``database/default/scoring/elec.yaml``: the
sigmoidal-dielectric global parameters, per residue / variant / atom partial
charges and the count-pair representative atoms, in file order, since later
representative lines override earlier ones) go to a second file.

Usage::

    python -m tmol_b200.chem.extract_db <tmol/database/default> <out.json> [<elec_out.json>]
"""

import json
import math
import sys

import yaml

CANONICAL = [
    "ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE",
    "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL",
]
EXTRA = ["HIS_D"]


def _deg(v):
    """Parse a '<float> deg' string (or a bare number, already degrees)."""
    if isinstance(v, str):
        v = v.strip()
        if v.endswith("deg"):
            v = v[: -len("deg")]
        return float(v)
    return float(v)


def extract(db_root):
    with open(f"{db_root}/chemical/chemical.yaml") as f:
        chem = yaml.safe_load(f)
    with open(f"{db_root}/scoring/ljlk.yaml") as f:
        ljlk = yaml.safe_load(f)
    with open(f"{db_root}/scoring/hbond.yaml") as f:
        hbond = yaml.safe_load(f)

    elements = {e["name"]: e["atomic_number"] for e in chem["element_types"]}
    ljlk_rows = {r["name"]: r for r in ljlk["atom_type_parameters"]}
    atom_types = []
    for at in chem["atom_types"]:
        row = ljlk_rows.get(at["name"])
        params = (
            [row[k] for k in ("lj_radius", "lj_wdepth", "lk_dgfree", "lk_lambda", "lk_volume")]
            if row is not None
            else [math.nan] * 5
        )
        atom_types.append(
            dict(
                name=at["name"],
                element=at["element"],
                is_hydrogen=bool(elements.get(at["element"], -1) == 1),
                is_donor=bool(at.get("is_donor", False)),
                is_acceptor=bool(at.get("is_acceptor", False)),
                is_hydroxyl=bool(at.get("is_hydroxyl", False)),
                is_polarh=bool(at.get("is_polarh", False)),
                acceptor_hybridization=at.get("acceptor_hybridization"),
                lj_radius=params[0],
                lj_wdepth=params[1],
                lk_dgfree=params[2],
                lk_lambda=params[3],
                lk_volume=params[4],
            )
        )

    residues = []
    by_name = {r["name"]: r for r in chem["residues"]}
    for name in CANONICAL + EXTRA:
        r = by_name[name]
        torsions = []
        for t in r.get("torsions", []):
            if not t["name"].startswith("chi"):
                continue
            if not all("atom" in t[k] for k in "abcd"):
                continue
            torsions.append(dict(name=t["name"], atoms=[t[k]["atom"] for k in "abcd"]))
        residues.append(
            dict(
                name=r["name"],
                base_name=r.get("base_name", r["name"]),
                name3=r.get("name3", r["name"]),
                one_letter_code=r.get("one_letter_code"),
                atoms=[[a["name"], a["atom_type"]] for a in r["atoms"]],
                atom_aliases=[[a["name"], a["alt_name"]] for a in r.get("atom_aliases", [])],
                bonds=[[b[0], b[1]] for b in r["bonds"]],
                connections=[[c["name"], c["atom"]] for c in r["connections"]],
                chis=torsions,
                icoors=[
                    [
                        ic["name"],
                        _deg(ic["phi"]),
                        _deg(ic["theta"]),
                        float(ic["d"]),
                        ic["parent"],
                        ic["grand_parent"],
                        ic["great_grand_parent"],
                    ]
                    for ic in r["icoors"]
                ],
                is_polymer=bool(r["properties"]["polymer"]["is_polymer"]),
            )
        )

    gp = ljlk["global_parameters"]
    global_params = {
        k: float(gp[k])
        for k in (
            "max_dis",
            "lj_dlin_sigma_factor",
            "lj_dlin_sigma_factor_soft",
            "lj_hbond_OH_donor_dis",
            "lj_hbond_hdis",
            "lj_hbond_dis",
            "lk_min_dis2sigma",
        )
    }
    lkball = {"lkb_water_dist": float(gp["lkb_water_dist"])}
    for k in ("lkb_water_angle_sp2", "lkb_water_angle_sp3", "lkb_water_angle_ring"):
        lkball[k] = math.radians(_deg(gp[k]))
    for k in ("lkb_water_tors_sp2", "lkb_water_tors_sp3", "lkb_water_tors_ring"):
        lkball[k] = [math.radians(_deg(v)) for v in gp[k]]
    return dict(
        source="tmol parameter database (chemical.yaml + scoring/ljlk.yaml + scoring/hbond.yaml)",
        atom_types=atom_types,
        residues=residues,
        ljlk_global_params=global_params,
        lkball_global_params=lkball,
        hbond_donor_atom_types=[x["d"] for x in hbond["donor_atom_types"]],
        hbond_acceptor_atom_types=[x["a"] for x in hbond["acceptor_atom_types"]],
    )


def extract_elec(db_root):
    with open(f"{db_root}/scoring/elec.yaml") as f:
        elec = yaml.safe_load(f)

    def res_var(tag):
        parts = tag.split(":")
        return parts[0], (parts[1] if len(parts) > 1 else "")

    charges = []
    for x in elec["atom_charge_parameters"]:
        res, var = res_var(x["res"])
        charges.append([res, var, x["atom"], float(x["charge"])])
    cp_reps = []
    for x in elec["atom_cp_reps_parameters"]:
        res, var = res_var(x["res"])
        cp_reps.append([res, var, x["atm_outer"], x["atm_inner"]])
    return dict(
        source="tmol parameter database (scoring/elec.yaml)",
        global_params={k: float(v) for k, v in elec["global_parameters"].items()},
        partial_charges=charges,
        cp_reps=cp_reps,
    )


def main(argv):
    db_root, out = argv[1], argv[2]
    data = extract(db_root)
    with open(out, "w") as f:
        json.dump(data, f, indent=0, sort_keys=False)
        f.write("\n")
    if len(argv) > 3:
        with open(argv[3], "w") as f:
            json.dump(extract_elec(db_root), f, indent=0, sort_keys=False)
            f.write("\n")


if __name__ == "__main__":
    main(sys.argv)
