"""Sliding-law and melange inputs for the drag tests (seeded, nodal).

The laws are CtrlVar.SlidingLaw's (BasalDrag.m:184-272): each case names the
law and fills the nodal fields it reads (F.q for Budd, F.muk for the Coulomb
family, F.V0 for Joughin); the melange case adds the ocean and atmosphere
velocity, drag and exponent fields (CtrlVar.IncludeMelangeModelPhysics).
"""
import numpy as np

LAWS = ["Weertman", "Budd", "Tsai", "Coulomb", "Cornford", "Umbi", "Joughin", "melange"]


def law_inputs(law, Nn, seed=0):
    """(CtrlVar.SlidingLaw, melange on/off, dict of nodal fields) for a case of LAWS."""
    rng = np.random.default_rng(seed)
    f = {}
    if law == "Budd":
        f["q"] = 1.0 + 0.1 * rng.random(Nn)
    if law in ("Tsai", "Coulomb", "Cornford", "Umbi"):
        # small enough that the Coulomb stress mu N is of the order of the Weertman stress, so the
        # Tsai minimum takes both branches and the regularised laws differ from either
        # (at least 0.008, so that the P2 interpolant, which undershoots the nodal minimum by up
        # to an eighth of the nodal range, stays positive at every integration point)
        f["muk"] = 0.008 + 0.014 * rng.random(Nn)
    if law == "Joughin":
        f["V0"] = 100.0 + 50.0 * rng.random(Nn)
    if law == "melange":
        f.update(uo=20 * rng.standard_normal(Nn), vo=5 * rng.standard_normal(Nn), Co=1e-2 + 0 * rng.random(Nn),
                 mo=3.0 + 0 * rng.random(Nn), ua=10 * rng.standard_normal(Nn), va=10 * rng.standard_normal(Nn),
                 Ca=1.0 + rng.random(Nn), ma=3.0 + 0 * rng.random(Nn))
        return "Weertman", True, f
    return law, False, f


def soften_C(P, power=0.2):
    """C of a synthetic problem pulled towards 1e-2 (C -> 1e-2 (C/1e-2)^power): on the coarse
    P2 test meshes the seeded C varies by two orders of magnitude between neighbouring nodes,
    so its P2 interpolant goes negative at integration points, where the reference's uvh drag
    (no C clamp, uvhAssemblyIntPointImplicitSUPG.m:78-79) is complex and the uv drag is clamped to
    Cmin.  Softened, C stays positive at every integration point."""
    P.C = 1e-2 * (P.C / 1e-2) ** power
    return P

