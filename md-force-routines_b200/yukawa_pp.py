"""Short-range (PP) part of the P3M force -- drop-in for the reference's
yukawa_pp.py (particle_particle, yukawa_pp.py:6-139), computed by the sm_100a
PP kernel of libp3m_b200."""
from p3m_b200.context import compat_context


def particle_particle(kappa, G, rc, Lv, pos, acc_s_r):
    """Linked-cell Yukawa-Ewald short-range sum -> (U_s_r, acc_s_r).

    Same arguments and results as yukawa_pp.py:6: ``acc_s_r`` (N,3) is
    overwritten with the PP acceleration and returned; Z is not used (unit
    charges, as in the reference). The cell grid is floor(L/rc) per side and
    must have at least 3 cells (with fewer the 27-cell stencil visits a pair
    twice); a smaller grid raises P3MError.
    """
    L = float(Lv[0])
    if not (float(Lv[1]) == L and float(Lv[2]) == L):
        raise ValueError("particle_particle: only cubic boxes are supported")
    ctx = compat_context(len(pos), L, kappa, G, rc)
    U, acc = ctx.pp(pos)
    acc_s_r[...] = acc
    return U, acc_s_r
